// ref_crlibm.cpp -- test infrastructure, NOT product code.
//
// The reference's torus computes its complex cube roots with the C library's
// atan2, sin/cos (fused by the compiler into sincos) and cbrt
// (volumes/kernel/TorusImplementation.h:283-316), whose last bits are the C
// library's own: glibc's cbrt is not correctly rounded.  libvgref_crlibm.so is
// the same reference build with the torus objects' calls to those three
// symbols redirected here, to correctly rounded versions (libvgb's crmath.cuh,
// compiled for the host).  Comparing the torus with both builds separates the
// rays whose result depends on the C library's rounding from the rest.
#include "../vecgeom_b200/csrc/crmath.cuh"

extern "C" {
double vgcr_atan2(double y, double x) { return vgb::cr_atan2(y, x); }
double vgcr_cbrt(double x) { return vgb::cr_cbrt(x); }
void vgcr_sincos(double x, double *s, double *c) { vgb::cr_sincos(x, s, c); }
}
