// refine.cuh -- the FP32+refine form of DistanceToIn/DistanceToOut: float
// arithmetic decides which surface the answer comes from, FP64 computes it.
//
// The reference's distance kernels are trees of decisions (is the point
// outside this surface, is the discriminant positive, does the hit point lie
// within the other surfaces' range, which candidate is nearer) that end in one
// closed-form root.  The FP32+refine form runs the decision tree in float and
// certifies each decision: every compared quantity carries a bound on its
// float error (computed alongside it from the magnitudes involved), and a
// decision counts only when its operands differ by more than their bounds.
// Then the float and the exact comparison agree, so the path taken is the FP64
// path, and the FP64 pass evaluates only the root that path ends in, with the
// reference's own operation order: the value is bit-identical to the FP64
// form's.  A point any of whose decisions is too close to call (near-surface
// points, grazing rays, long rays whose float roots lose their digits) takes
// the whole FP64 kernel instead.  Error of the form: 0 for every point, by
// construction; what the float pass buys is the decision work done at float
// throughput and the FP64 work cut to one root per point.
//
// Error bounds: u = 2^-24 (float unit roundoff); the inputs are rounded to
// float (relative error u).  Bounds are first-order in u and multiplied by a
// safety factor kSafe; the FP64 kernels' own rounding (2^-53) is far below them.
#pragma once
#include "batch.cuh"

namespace vgb {

constexpr float kU = 5.9604645e-08f;  // 2^-24
constexpr float kSafe = 8.f;

// Certification of float decisions: a comparison of a and b whose error bound
// is e marks the point uncertain unless |a - b| > e (NaN operands included).
struct Cert {
  bool ok = true;
  VGB_HD bool gt(float a, float b, float e) {
    ok &= fabsf(a - b) > e;
    return a > b;
  }
  VGB_HD bool ge(float a, float b, float e) {
    ok &= fabsf(a - b) > e;
    return a >= b;
  }
  VGB_HD bool lt(float a, float b, float e) { return gt(b, a, e); }
  VGB_HD bool le(float a, float b, float e) { return ge(b, a, e); }
};

// A float value with a bound on its absolute error.
struct FE {
  float v, e;
};

// ---------------------------------------------------------------------------
// Sphere DistanceToIn (USolids USphere::DistanceToIn, USphere.cc:630-1563, as
// SphereOps::dti_core restates it).  Full-phi spheres; a sphere with a phi
// section runs the FP64 kernel for every point.
// ---------------------------------------------------------------------------
enum SphereDtiWinner : int {
  kSdUncertain = 0,
  kSdInf,
  kSdZero,
  kSdOuter,    // -b - sqrt(d2) on rmax
  kSdInner,    // -b + sqrt(d2) on rmin
  kSdSMinus,   // start theta cone, -b - d
  kSdSPlus,    // start theta cone, -b + d
  kSdEMinus,   // end theta cone, -b - d
  kSdEPlus,    // end theta cone, -b + d
};

struct SphereRefine {
  // theta of (rho, z) against cut k: -1 below, +1 above; certified margin on
  // f = z sin c - rho cos c = r sin(c - theta), whose float error is bounded
  // from the errors of rho and z.
  static VGB_HD int cut_side_f(const ThetaCut &k, FE rho, FE z, Cert &ct) {
    if (k.mode == 1) return 1;
    if (k.mode == 2) return -1;
    const float sn = (float)k.sn, cs = (float)k.cs;
    const float f = z.v * sn - rho.v * cs;
    const float e = kSafe * (fabsf(sn) * z.e + fabsf(cs) * rho.e +
                             3.f * kU * (fabsf(z.v) + rho.v));
    ct.ok &= fabsf(f) > e;
    return f > 0.f ? -1 : 1;
  }
  static VGB_HD bool theta_in(const SphereP &s, FE rho, FE z, Cert &ct) {
    // th >= tolS && th <= tolE
    return cut_side_f(s.cut[kCutTolS], rho, z, ct) > 0 && cut_side_f(s.cut[kCutTolE], rho, z, ct) < 0;
  }

  // One theta cone, in FP64 with dti_core's operation order: its discriminant
  // is ill-conditioned (for a cut at pi/2 the "cone" is the plane z = 0 with
  // tan^2 ~ 2.7e32, and b^2 - c cancels to a few ulp), so float cannot decide
  // it.  Returns whether d2 >= 0 (and t1 != 0) and both roots.
  struct Cone64 {
    bool real;
    double minus, plus;
  };
  static VGB_HD Cone64 cone64(double tan2, double dist2, double pDotV2d, const V3<double> &p,
                             const V3<double> &v) {
    Cone64 o = {false, 0., 0.};
    const double t1 = 1. - v.z * v.z * (1. + tan2);
    const double t2 = pDotV2d - p.z * v.z * tan2;
    if (t1 != 0) {
      const double b = t2 / t1;
      const double c = dist2 / t1;
      const double d2 = b * b - c;
      if (d2 >= 0) {
        const double d = sqrt(d2);
        o.real = true;
        o.minus = -b - d;
        o.plus = -b + d;
      }
    }
    return o;
  }

  // The winner of DistanceToIn for this point, or kSdUncertain.
  static VGB_HD int select(const SphereP &s, const V3<double> &p64, const V3<double> &v64) {
    if (!s.fullPhi) return kSdUncertain;
    Cert ct;
    const float px = (float)p64.x, py = (float)p64.y, pz = (float)p64.z;
    const float vx = (float)v64.x, vy = (float)v64.y, vz = (float)v64.z;
    const float fRmin = (float)s.rmin, fRmax = (float)s.rmax;
    const float rho2 = px * px + py * py;
    const float rad2 = rho2 + pz * pz;
    const float pDotV2d = px * vx + py * vy;
    const float pDotV3d = pDotV2d + pz * vz;
    const float r = sqrtf(rad2);
    // error bounds of the point quantities
    const FE Rad2 = {rad2, kSafe * 5.f * kU * rad2};
    const FE B2 = {pDotV2d, kSafe * 4.f * kU * sqrtf(rho2)};
    const FE B = {pDotV3d, kSafe * 5.f * kU * r};
    const FE Pz = {pz, kU * fabsf(pz)};
    const FE Rho = {sqrtf(rho2), kSafe * 3.f * kU * sqrtf(rho2)};
    const float tolORMax2 = (float)((s.rmax + s.mkTolerance * 0.5) * (s.rmax + s.mkTolerance * 0.5));
    const float tolIRMax2 = (float)((s.rmax - s.mkTolerance * 0.5) * (s.rmax - s.mkTolerance * 0.5));
    const double hrt = s.rminTolerance * 0.5;
    const float tolORMin2 = (float)(s.rmin > hrt ? (s.rmin - hrt) * (s.rmin - hrt) : 0.0);
    const float tolIRMin2 = (float)((s.rmin + hrt) * (s.rmin + hrt));
    const float eTol2 = kSafe * 2.f * kU * (float)(s.rmax * s.rmax);  // rounding of the tolerances
    const float halfRminTol = (float)hrt;
    const float dRmax = 100.f * fRmax;
    const float mkTolR = (float)(s.mkTolerance * s.rmax);
    // the point's polar angle against the cuts
    auto p_side = [&](int cut) { return cut_side_f(s.cut[cut], Rho, Pz, ct); };
    auto strictly_theta = [&]() { return p_side(kCutTolS2) > 0 && p_side(kCutTolE2) < 0; };
    // hit point of a root sd (float value and bound)
    auto hit = [&](FE sd, FE &rhoi, FE &zi, FE &radi2) {
      const float xi = px + sd.v * vx, yi = py + sd.v * vy, z = pz + sd.v * vz;
      const float eh = kSafe * (sd.e + 2.f * kU * (fabsf(px) + fabsf(py) + fabsf(pz) + 2.f * fabsf(sd.v)));
      const float rh2 = xi * xi + yi * yi;
      rhoi = {sqrtf(rh2), eh * 2.f + kSafe * 2.f * kU * sqrtf(rh2)};
      zi = {z, eh};
      radi2 = {rh2 + z * z, kSafe * (2.f * sqrtf(rh2 + z * z) * 2.f * eh + 4.f * kU * (rh2 + z * z))};
    };

    // outer sphere (:667-760)
    const float c = rad2 - fRmax * fRmax;
    const float e_c = Rad2.e + kSafe * 2.f * kU * (rad2 + fRmax * fRmax);
    const float d2 = pDotV3d * pDotV3d - c;
    const float e_d2 = kSafe * (2.f * fabsf(pDotV3d) * B.e + e_c + 2.f * kU * (pDotV3d * pDotV3d + fabsf(c)));
    if (ct.gt(c, mkTolR, e_c)) {
      if (ct.ge(d2, 0.f, e_d2)) {
        const float sq = sqrtf(d2);
        const FE sd = {-pDotV3d - sq, B.e + kSafe * (e_d2 / fmaxf(sq, 1e-30f) + 2.f * kU * (fabsf(pDotV3d) + sq))};
        if (ct.ge(sd.v, 0.f, sd.e)) {
          if (!ct.le(sd.v, dRmax, sd.e + kU * dRmax)) return kSdUncertain;  // split path: FP64
          if (s.fullTheta) return ct.ok ? kSdOuter : kSdUncertain;
          FE rhoi, zi, radi2;
          hit(sd, rhoi, zi, radi2);
          if (theta_in(s, rhoi, zi, ct)) return ct.ok ? kSdOuter : kSdUncertain;
        }
      } else {
        return ct.ok ? kSdInf : kSdUncertain;
      }
    } else {
      if (ct.gt(rad2, tolIRMax2, Rad2.e + eTol2) && ct.ge(d2, mkTolR, e_d2) &&
          ct.lt(pDotV3d, 0.f, B.e)) {
        if (s.fullTheta) return ct.ok ? kSdZero : kSdUncertain;
        if (strictly_theta()) return ct.ok ? kSdZero : kSdUncertain;
      }
    }
    if (!ct.ok) return kSdUncertain;

    int win = kSdInf;
    FE snxt = {HUGE_VALF, 0.f};
    // inner sphere (:790-930)
    if (s.rmin != 0) {
      const float ci = rad2 - fRmin * fRmin;
      const float e_ci = Rad2.e + kSafe * 2.f * kU * (rad2 + fRmin * fRmin);
      const float d2i = pDotV3d * pDotV3d - ci;
      const float e_d2i = kSafe * (2.f * fabsf(pDotV3d) * B.e + e_ci + 2.f * kU * (pDotV3d * pDotV3d + fabsf(ci)));
      const bool on_inner = ct.gt(ci, -halfRminTol, e_ci) && ct.lt(rad2, tolIRMin2, Rad2.e + eTol2) &&
                            (ct.lt(d2i, fRmin * (float)kTolerance, e_d2i) || ct.ge(pDotV3d, 0.f, B.e));
      if (!ct.ok) return kSdUncertain;
      if (on_inner) {
        if (s.fullTheta) return kSdZero;
        if (strictly_theta()) return ct.ok ? kSdZero : kSdUncertain;
      } else if (ct.ge(d2i, 0.f, e_d2i)) {
        const float sq = sqrtf(d2i);
        const FE sd = {-pDotV3d + sq, B.e + kSafe * (e_d2i / fmaxf(sq, 1e-30f) + 2.f * kU * (fabsf(pDotV3d) + sq))};
        if (ct.ge(sd.v, halfRminTol, sd.e)) {
          if (s.fullTheta) {
            snxt = sd;
            win = kSdInner;
          } else {
            FE rhoi, zi, radi2;
            hit(sd, rhoi, zi, radi2);
            if (theta_in(s, rhoi, zi, ct)) {
              snxt = sd;
              win = kSdInner;
            }
          }
        }
      }
      if (!ct.ok) return kSdUncertain;
    }
    if (s.fullTheta) return win;

    // theta cones (:1044-1560): candidates in FP64 (cone64), their hit-point
    // tests and the comparison with the running minimum in float
    const double rho2_64 = p64.x * p64.x + p64.y * p64.y;
    const double pDotV2d_64 = p64.x * v64.x + p64.y * v64.y;
    const bool haveS = s.stheta != 0, haveE = s.eTheta < kPi;
    const double dist2S = haveS ? rho2_64 - p64.z * p64.z * s.tanSTheta2 : 0.;
    const double dist2E = haveE ? rho2_64 - p64.z * p64.z * s.tanETheta2 : 0.;
    // accept(sd, thetaC): the hit point within the radial shell and on the
    // cone's side (zi * (thetaC - pi/2) <= 0, exactly true when thetaC = pi/2)
    auto accept = [&](double sd64, double thetaC, int w) {
      const FE sd = {(float)sd64, kU * fabsf((float)sd64)};
      FE rhoi, zi, radi2;
      hit(sd, rhoi, zi, radi2);
      const double tc = thetaC - kPi / 2;
      bool side_ok = true;
      if (tc != 0) {
        const float side = zi.v * (float)tc;
        side_ok = ct.le(side, 0.f, kSafe * (zi.e * fabsf((float)tc) + kU * fabsf(side)));
      }
      if (ct.le(radi2.v, tolORMax2, radi2.e + eTol2) && ct.ge(radi2.v, tolORMin2, radi2.e + eTol2) &&
          side_ok) {
        snxt = sd;
        win = w;
      }
    };
    // sd >= 0 && sd < snxt, sd exact (FP64), snxt within its bound
    auto admissible = [&](double sd64) {
      if (!(sd64 >= 0)) return false;
      return ct.lt((float)sd64, snxt.v, kU * fabsf((float)sd64) + snxt.e);
    };
    // the first root of a cone the point is outside of: -b - d, or -b + d when
    // that is negative or on the cone's far nappe (zi * (theta - pi/2) > 0)
    auto first_root = [&](const Cone64 &k, double thetaC, int wm, int wp, double &sd, int &w) {
      sd = k.minus;
      w = wm;
      const double zi = p64.z + sd * v64.z;
      if ((sd < 0) || (zi * (thetaC - kPi / 2) > 0)) {
        sd = k.plus;
        w = wp;
      }
    };
    if (p_side(kCutTolS) < 0) {
      if (!haveS) return kSdUncertain;  // unreachable: no cut below theta = 0
      const Cone64 k = cone64(s.tanSTheta2, dist2S, pDotV2d_64, p64, v64);
      if (k.real) {
        double sd;
        int w;
        first_root(k, s.stheta, kSdSMinus, kSdSPlus, sd, w);
        if (admissible(sd)) accept(sd, s.stheta, w);
      }
      if (haveE) {
        const Cone64 k2 = cone64(s.tanETheta2, dist2E, pDotV2d_64, p64, v64);
        if (k2.real && admissible(k2.plus)) accept(k2.plus, s.eTheta, kSdEPlus);
      }
    } else if (p_side(kCutTolE) > 0) {
      if (!haveE) return kSdUncertain;  // unreachable: no cut above theta = pi
      const Cone64 k = cone64(s.tanETheta2, dist2E, pDotV2d_64, p64, v64);
      if (k.real) {
        double sd;
        int w;
        first_root(k, s.eTheta, kSdEMinus, kSdEPlus, sd, w);
        if (admissible(sd)) accept(sd, s.eTheta, w);
      }
      if (haveS) {
        const Cone64 k2 = cone64(s.tanSTheta2, dist2S, pDotV2d_64, p64, v64);
        if (k2.real && admissible(k2.plus)) accept(k2.plus, s.stheta, kSdSPlus);
      }
    } else if (p_side(kCutTolS2) < 0 && s.stheta > 0.5 * kAngTolerance) {
      return kSdUncertain;  // on the start cone: the FP64 path
    } else if (p_side(kCutTolE2) > 0 && s.eTheta < kPi - kAngTolerance) {
      return kSdUncertain;  // on the end cone: the FP64 path
    } else {
      // a missing cone has dist2 = inf: c = +-inf makes d2 = -inf or gives the
      // root +inf, neither below snxt, so it never yields a candidate
      if (haveS) {
        const Cone64 k = cone64(s.tanSTheta2, dist2S, pDotV2d_64, p64, v64);
        if (k.real && admissible(k.plus)) accept(k.plus, s.stheta, kSdSPlus);
      }
      if (haveE) {
        const Cone64 k = cone64(s.tanETheta2, dist2E, pDotV2d_64, p64, v64);
        if (k.real && admissible(k.plus)) accept(k.plus, s.eTheta, kSdEPlus);
      }
    }
    return ct.ok ? win : kSdUncertain;
  }

  // The FP64 value of a winner, in dti_core's operation order.
  static VGB_HD double eval(const SphereP &s, const V3<double> &p, const V3<double> &v, int win) {
    using R = double;
    const R rho2 = p.x * p.x + p.y * p.y;
    const R rad2 = rho2 + p.z * p.z;
    const R pDotV2d = p.x * v.x + p.y * v.y;
    const R pDotV3d = pDotV2d + p.z * v.z;
    switch (win) {
    case kSdInf: return Lim<R>::inf();
    case kSdZero: return 0.;
    case kSdOuter: {
      const R fRmax = s.rmax;
      const R c = rad2 - fRmax * fRmax;
      const R d2 = pDotV3d * pDotV3d - c;
      return -pDotV3d - sqrt(d2);
    }
    case kSdInner: {
      const R fRmin = s.rmin;
      const R c = rad2 - fRmin * fRmin;
      const R d2 = pDotV3d * pDotV3d - c;
      return -pDotV3d + sqrt(d2);
    }
    default: {
      const bool start = (win == kSdSMinus || win == kSdSPlus);
      const R tan2 = start ? s.tanSTheta2 : s.tanETheta2;
      const R dist2 = start ? ((s.stheta != 0) ? rho2 - p.z * p.z * tan2 : Lim<R>::inf())
                            : ((s.eTheta < kPi) ? rho2 - p.z * p.z * tan2 : Lim<R>::inf());
      const R t1 = (R)1 - v.z * v.z * ((R)1 + tan2);
      const R t2 = pDotV2d - p.z * v.z * tan2;
      const R b = t2 / t1;
      const R c = dist2 / t1;
      const R d2 = b * b - c;
      const R d = sqrt(d2);
      return (win == kSdSMinus || win == kSdEMinus) ? -b - d : -b + d;
    }
    }
  }
};

}  // namespace vgb

// ---------------------------------------------------------------------------
// The FP32+refine batch kernel for DistanceToIn.  A block works through tiles
// of kRefineTile points: every thread selects in float and, when its point is
// certified, writes the FP64 value of the winning root; uncertain points are
// appended to a block queue (warp-aggregated) and, once the tile is done, the
// block runs the FP64 kernel's DistanceToIn on the queue with every lane busy.
// ---------------------------------------------------------------------------
namespace vgb {

constexpr int kRefineBlock = 256;
constexpr int kRefineTile = 1024;

// points certified / sent to the FP64 path, summed over all FP32+refine
// launches since the last reset (vgb_refine_counts; one translation unit,
// batch_f64.cu, includes this header)
struct RefineCounts {
  unsigned long long certified, fallback;
};
static __device__ RefineCounts g_refine_counts;

template <class Ops> struct RefineDti {
  using type = void;
};
template <> struct RefineDti<SphereOps<double>> {
  using type = SphereRefine;
};

template <class Rf, class Ops, class P>
__global__ void __launch_bounds__(kRefineBlock)
    k_refine_dti(const P prm, const DXform X, const BatchIO io) {
  __shared__ int32_t queue[kRefineTile];
  __shared__ int32_t qn;
  double *out = static_cast<double *>(io.out);
  const int lane = threadIdx.x & 31;
  unsigned long long certified = 0;
  for (int64_t base = (int64_t)blockIdx.x * kRefineTile; base < io.n;
       base += (int64_t)gridDim.x * kRefineTile) {
    if (threadIdx.x == 0) qn = 0;
    __syncthreads();
    for (int j = 0; j < kRefineTile / kRefineBlock; ++j) {
      const int64_t i = base + j * kRefineBlock + threadIdx.x;
      bool fb = false;
      if (i < io.n) {
        const V3<double> m = {__ldg(io.x + i), __ldg(io.y + i), __ldg(io.z + i)};
        const V3<double> d = {__ldg(io.dx + i), __ldg(io.dy + i), __ldg(io.dz + i)};
        const V3<double> p = xf_point(X, m), v = dti_dir<Ops>(X, d);
        const int w = Rf::select(prm, p, v);
        if (w) {
          out[i] = Rf::eval(prm, p, v, w);
          ++certified;
        } else {
          fb = true;
        }
      }
      const unsigned mask = __ballot_sync(0xffffffffu, fb);
      if (mask) {
        const int leader = __ffs(mask) - 1;
        int pos = 0;
        if (lane == leader) pos = atomicAdd(&qn, __popc(mask));
        pos = __shfl_sync(0xffffffffu, pos, leader);
        if (fb) queue[pos + __popc(mask & ((1u << lane) - 1u))] = (int32_t)(i - base);
      }
    }
    __syncthreads();
    const int q = qn;
    for (int k = threadIdx.x; k < q; k += kRefineBlock) {
      const int64_t i = base + queue[k];
      const V3<double> m = {__ldg(io.x + i), __ldg(io.y + i), __ldg(io.z + i)};
      const V3<double> d = {__ldg(io.dx + i), __ldg(io.dy + i), __ldg(io.dz + i)};
      out[i] = Ops::distance_to_in(prm, xf_point(X, m), dti_dir<Ops>(X, d), __ldg(io.step + i));
    }
    if (threadIdx.x == 0 && q) atomicAdd(&g_refine_counts.fallback, (unsigned long long)q);
    __syncthreads();
  }
  // one atomic per warp for the certified count
  for (int o = 16; o; o >>= 1) certified += __shfl_down_sync(0xffffffffu, certified, o);
  if (lane == 0 && certified) atomicAdd(&g_refine_counts.certified, certified);
}

}  // namespace vgb
