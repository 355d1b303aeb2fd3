// wedge.cuh -- the phi-section helper shared by tube, cone, torus and polycone
// (volumes/Wedge.h:42-330, source/Wedge.cpp:14-45).
#pragma once
#include "vgb_core.cuh"

namespace vgb {

// Wedge(angle = dphi, zeroangle = sphi); the along/normal vectors are computed
// on the host with the same std::cos/std::sin calls as the reference.
struct WedgeP {
  double a1x, a1y, a2x, a2y;  // along vectors of the two half-planes
  double n1x, n1y, n2x, n2y;  // inward normals
  double dphi;
  int32_t lt_pi;  // fDPhi < kPi
  int32_t pad;
};

template <class R> struct WedgeOps {
  // Wedge::IsOnSurfaceGeneric (volumes/Wedge.h:225-237)
  static VGB_HD bool on_surface(double ax, double ay, double nx, double ny, R x, R y) {
    const bool c1 = (R)ax * x + (R)ay * y >= (R)0.;
    if (!c1) return false;
    return fabs((R)nx * x + (R)ny * y) < (R)kTolerance;
  }

  // Wedge::GenericKernelForContainsAndInside (volumes/Wedge.h:190-222)
  template <bool ForInside>
  static VGB_HD void contains_inside(const WedgeP &w, R x, R y, bool &cin, bool &cout) {
    const R startCheck = (-x * (R)w.a1y + y * (R)w.a1x);
    const R endCheck = (-(R)w.a2x * y + (R)w.a2y * x);
    cout = startCheck < (R)0.;
    if (w.lt_pi)
      cout |= endCheck < (R)0.;
    else
      cout &= endCheck < (R)0.;
    if (ForInside) {
      const bool onSurface =
          on_surface(w.a1x, w.a1y, w.n1x, w.n1y, x, y) || on_surface(w.a2x, w.a2y, w.n2x, w.n2y, x, y);
      cout &= !onSurface;
      cin = !onSurface && !cout;
    }
  }

  // Wedge::ContainsWithBoundary (volumes/Wedge.h:164-172)
  static VGB_HD bool contains_with_boundary(const WedgeP &w, R x, R y) {
    bool ci, co;
    contains_inside<true>(w, x, y, ci, co);
    return !co;
  }

  // Wedge::SafetyToOut (volumes/Wedge.h:242-264)
  static VGB_HD R safety_to_out(const WedgeP &w, R x, R y) {
    const R d1 = x * (R)w.n1x + y * (R)w.n1y;
    const R d2 = x * (R)w.n2x + y * (R)w.n2y;
    if (w.lt_pi) return vmin(d1, d2);
    return vmax(d1, d2);
  }

  // Wedge::SafetyToIn (volumes/Wedge.h:268-290)
  static VGB_HD R safety_to_in(const WedgeP &w, R x, R y) {
    const R d1 = x * (R)w.n1x + y * (R)w.n1y;
    const R d2 = x * (R)w.n2x + y * (R)w.n2y;
    const R m1 = (R)-1 * d1, m2 = (R)-1 * d2;
    if (w.lt_pi) return vmax(m1, m2);
    return vmin(m1, m2);
  }
};

}  // namespace vgb
