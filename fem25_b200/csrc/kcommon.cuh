// Device helpers shared by the kernels: complex arithmetic in the forms the
// reference writes, the per-quadrature-point geometry of CJMK_TVI / CJACCQ
// (cjac.f:1-138, 399-581) and the PML stretching function ZDAMPFN
// (cjac.f:818-921).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "ctx.cuh"

namespace fem25 {

struct dcx {
  double re, im;
};
__host__ __device__ __forceinline__ dcx zadd(dcx a, dcx b) { return dcx{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ dcx zsub(dcx a, dcx b) { return dcx{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ dcx zmul(dcx a, dcx b) {
  return dcx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// (a+ib)/(c+id), textbook form
__host__ __device__ __forceinline__ dcx zdiv(dcx a, dcx b) {
  double den = b.re * b.re + b.im * b.im;
  return dcx{(a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den};
}
// Fortran X**2 (integer power): (1*x)*x
__host__ __device__ __forceinline__ double ipow2(double x) {
  double r = 1.0;
  r = r * x;
  r = r * x;
  return r;
}

// ZDAMPFN: 1 / (kappa + |d| / (alpha + i omega)), d = dmax (rn/delta)^2,
// dmax = -3 Vp ln(R) / (2 delta) unless overridden, alpha = pi fc (1 - rn/delta)
__device__ __forceinline__ dcx zdampfn(double rn, double vp, double delta, double dmax_in,
                                       double logr, double rkappa, double fcent, double omega) {
  double dmax;
  if (dmax_in > 0.0) dmax = dmax_in;
  else dmax = -3.0 * vp * logr / (2.0 * delta);
  double d = dmax * ipow2(rn / delta);
  double alpha = 3.1415926535897931 * fcent * (1.0 - rn / delta);
  dcx z = zadd(dcx{rkappa, 0.0}, zdiv(dcx{fabs(d), 0.0}, dcx{alpha, omega}));
  return zdiv(dcx{1.0, 0.0}, z);
}

struct QGeo {
  double dxdxi, dxdeta, dzdxi, dzdeta, rjac, lam, mu, rho, xdep, zdep, vel;
};

// Geometry and interpolated model at quadrature point q of an element with
// anchors ie (1-based).  Returns false when the Jacobian is undefined or
// negative (the reference's IERR=1 branch).
__device__ __forceinline__ bool quad_geo(const MeshView &mv, const DevTables &dt, int4 ie, int q,
                                         bool pml, QGeo &g) {
  const double *sf = dt.sf + 4 * q;
  const double *dsx = dt.dsf + 8 * q;      // d/dxi of the 4 anchor functions
  const double *dse = dt.dsf + 8 * q + 4;  // d/deta
  const int il[4] = {ie.x - 1, ie.y - 1, ie.z - 1, ie.w - 1};
  double x = 0.0, z = 0.0, d1 = 0.0, d2 = 0.0, r = 0.0;
  double xdep = 0.0, zdep = 0.0, vel = 0.0;
  double dxdxi = 0.0, dxdeta = 0.0, dzdxi = 0.0, dzdeta = 0.0;
#pragma unroll
  for (int ia = 0; ia < 4; ia++) {
    const int p = il[ia];
    const double xa = mv.x[p], za = mv.z[p], la = mv.lam[p], ma = mv.mu[p], ra = mv.rho[p];
    x = x + sf[ia] * xa;
    z = z + sf[ia] * za;
    d1 = d1 + sf[ia] * la;
    d2 = d2 + sf[ia] * ma;
    r = r + sf[ia] * ra;
    if (pml) {
      xdep = xdep + sf[ia] * mv.xd[p];
      zdep = zdep + sf[ia] * mv.zd[p];
      double alpha2 = (la + 2.0 * ma) / ra;
      vel = vel + sf[ia] * sqrt(alpha2);
    }
    dxdxi = dxdxi + dsx[ia] * xa;
    dxdeta = dxdeta + dse[ia] * xa;
    dzdxi = dzdxi + dsx[ia] * za;
    dzdeta = dzdeta + dse[ia] * za;
  }
  (void)x;
  (void)z;
  g.dxdxi = dxdxi;
  g.dxdeta = dxdeta;
  g.dzdxi = dzdxi;
  g.dzdeta = dzdeta;
  g.lam = d1;
  g.mu = d2;
  g.rho = r;
  g.xdep = xdep;
  g.zdep = zdep;
  g.vel = vel;
  double rjac = dxdxi * dzdeta - dxdeta * dzdxi;
  g.rjac = rjac;
  return !(fabs(rjac) <= 2.22e-16 || rjac < 0.0);
}

}  // namespace fem25
