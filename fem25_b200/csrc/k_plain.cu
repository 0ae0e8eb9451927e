// Plain per-(omega, py) FP64 assembly: one CTA per element builds the 75x75
// element matrix exactly as KM25ISOQ / CM25ISOQ do (estiff25.f:1-334), then a
// gather kernel replays the element-to-nonzero map and sums the contributions
// of every nonzero in element order (ASMBLE_CDIST, asmble.f90:235-314).
//
// This translation unit is compiled with -fmad=false: every multiply and add
// is rounded separately, in the order the reference writes them, so the FP64
// sums are the reference arithmetic without FMA contraction.  It is compiled
// a second time with FEM25_PLAIN_FMA defined and FMA contraction allowed,
// into the nested namespace fem25::plain_fma, for launch_elem_plain_fma (the
// same element kernels with fused multiply-adds, a benchmark option of
// fem25_assemble_dev).
#include <cub/device/device_scan.cuh>

#include "ctx.cuh"
#include "kcommon.cuh"

#ifdef FEM25_PLAIN_FMA
namespace fem25 {
namespace plain_fma {
#else
namespace fem25 {
#endif

struct PlainArgs {
  double w2, py2, wpy, omega;
  PmlParams pml;
  double logr;  // log(RCOEFF) evaluated on the host
  // dispersive media (KMDAMP / CMDAMP)
  int ldisp;
  double freq0;
  double fac1;  // log(FREQ / FREQ0) evaluated on the host (VCMPLX, haskattn.f:633)
  int ebase;    // element of block 0 (launches over an element range)
};

// VCMPLX (haskattn.f:602-646): complex velocity of Aki & Richards 5.94,
// v (1 + ln(f/f0) / (pi Q)) - i v / (2 Q); Q = 9999 or f0 = 0 mean none
__device__ __forceinline__ dcx vcmplx(const PlainArgs &pa, double v, double q) {
  if (pa.freq0 == 0.0 || fabs(q - 9999.0) < 1.0e-5) return dcx{v, 0.0};
  if (q == 0.0) return dcx{v, 0.0};
  double fact = 1.0 + 1.0 / (3.1415926535897931 * q) * pa.fac1;
  if (fact < 0.1) fact = 0.1;
  return dcx{v * fact, -v / (2.0 * q)};
}

// CJKM_QUAL / CJCM_QUAL (cjac.f:142-278, 585-755): interpolated Vp, Vs
// (velocities, not moduli) and quality factors at point q
__device__ __forceinline__ void quad_qual(const MeshView &mv, const DevTables &dt, int4 ie, int q,
                                          double &vp, double &vs, double &qpp, double &qss) {
  const double *sf = dt.sf + 4 * q;
  const int il[4] = {ie.x - 1, ie.y - 1, ie.z - 1, ie.w - 1};
  vp = 0.0;
  vs = 0.0;
  qpp = 0.0;
  qss = 0.0;
#pragma unroll
  for (int ia = 0; ia < 4; ia++) {
    const int p = il[ia];
    const double la = mv.lam[p], ma = mv.mu[p], ra = mv.rho[p];
    double vpp = sqrt((la + 2.0 * ma) / ra);
    double vss = sqrt(ma / ra);
    vp = vp + sf[ia] * vpp;
    vs = vs + sf[ia] * vss;
    qpp = qpp + sf[ia] * mv.qp[p];
    qss = qss + sf[ia] * mv.qs[p];
  }
}

// shared-memory layout of the element kernel (doubles)
constexpr int kSmShx = 0;
constexpr int kSmShz = kSmShx + kNq * kNen;
constexpr int kSmShn = kSmShz + kNq * kNen;
constexpr int kSmQ = kSmShn + kNq * kNen;   // per-quadrature-point coefficients
constexpr int kNqc = 17;                    // coefficient slots per point
constexpr int kSmTot = kSmQ + kNqc * kNq;
constexpr int kPlainThreads = 640;

// KMDAMP (estiff25.f:511-752) for the node pair (IAE = a, IBE = b): the
// density-normalised operator with complex velocities; the imaginary mass
// terms go into KE; output ME + Re(KE), Im(KE) as ASMBLE_CDIST adds them
__device__ __forceinline__ void kmdamp_pair(const double *qc, const double *shx, const double *shz,
                                            const double *shn, int a, int b, double wpy,
                                            double2 *out) {
  double me0 = 0.0, me1 = 0.0, me2 = 0.0;
  dcx ke[9];
#pragma unroll
  for (int k = 0; k < 9; k++) ke[k] = dcx{0.0, 0.0};
  for (int intx = 0; intx < kNint; intx++)
    for (int intz = 0; intz < kNint; intz++) {
      const int q = intx + kNint * intz;
      const double *c = qc + kNqc * q;
      const double rvp2 = c[5], qvp2 = c[6], rvs2 = c[7], qvs2 = c[8];
      const double rm1 = c[9], qm1 = c[10], rm2 = c[11], qm2 = c[12];
      const double phib = shn[q * kNen + b], phibx = shx[q * kNen + b], phibz = shz[q * kNen + b];
      const double phia = shn[q * kNen + a], phiax = shx[q * kNen + a], phiaz = shz[q * kNen + a];
      const double rm11t1 = rm1 * phib, qm11t1 = qm1 * phib;
      const double rm22t1 = rm2 * phib, qm22t1 = qm2 * phib;
      const double rk11t1 = rvp2 * phibx, qk11t1 = qvp2 * phibx;
      const double rk11t2 = rvs2 * phibz, qk11t2 = qvs2 * phibz;
      const double rk13t1 = rvp2 * phibz, qk13t1 = qvp2 * phibz;
      const double rk13t2 = rvs2 * phibx, qk13t2 = qvs2 * phibx;
      const double rk13t3 = -(2.0 * rvs2 * phibz), qk13t3 = -(2.0 * qvs2 * phibz);
      const double rk22t1 = rvs2 * phibx, qk22t1 = qvs2 * phibx;
      const double rk22t2 = rvs2 * phibz, qk22t2 = qvs2 * phibz;
      const double rk31t1 = rvp2 * phibx, qk31t1 = qvp2 * phibx;
      const double rk31t2 = rvs2 * phibz, qk31t2 = qvs2 * phibz;
      const double rk31t3 = -(2.0 * rvs2 * phibx), qk31t3 = -(2.0 * qvs2 * phibx);
      const double rk33t1 = rvp2 * phibz, qk33t1 = qvp2 * phibz;
      const double rk33t2 = rvs2 * phibx, qk33t2 = qvs2 * phibx;
      const double rk12t1 = wpy * rvp2 * phib, qk12t1 = wpy * qvp2 * phib;
      const double rk12t2 = -(2.0 * wpy * rvs2 * phib), qk12t2 = -(2.0 * wpy * qvs2 * phib);
      const double rk12t3 = -(wpy * rvs2 * phibx), qk12t3 = -(wpy * qvs2 * phibx);
      const double rk21t1 = wpy * rvp2 * phibx, qk21t1 = wpy * qvp2 * phibx;
      const double rk21t2 = -(2.0 * wpy * rvs2 * phibx), qk21t2 = -(2.0 * wpy * qvs2 * phibx);
      const double rk21t3 = -(wpy * rvs2 * phib), qk21t3 = -(wpy * qvs2 * phib);
      const double rk23t1 = wpy * rvp2 * phibz, qk23t1 = wpy * qvp2 * phibz;
      const double rk23t2 = -(2.0 * wpy * rvs2 * phibz), qk23t2 = -(2.0 * wpy * qvs2 * phibz);
      const double rk23t3 = -(wpy * rvs2 * phib), qk23t3 = -(wpy * qvs2 * phib);
      const double rk32t1 = wpy * rvp2 * phib, qk32t1 = wpy * qvp2 * phib;
      const double rk32t2 = -(2.0 * wpy * rvs2 * phib), qk32t2 = -(2.0 * wpy * qvs2 * phib);
      const double rk32t3 = -(wpy * rvs2 * phibz), qk32t3 = -(wpy * qvs2 * phibz);
      const double rme11 = rm11t1 * phia, qme11 = qm11t1 * phia;
      const double rme22 = rm22t1 * phia, qme22 = qm22t1 * phia;
      const double rme33 = rme11, qme33 = qme11;
      const double rke11 = rk11t1 * phiax + rk11t2 * phiaz;
      const double qke11 = qk11t1 * phiax + qk11t2 * phiaz;
      const double rke13 = rk13t1 * phiax + rk13t2 * phiaz + rk13t3 * phiax;
      const double qke13 = qk13t1 * phiax + qk13t2 * phiaz + qk13t3 * phiax;
      const double rke22 = rk22t1 * phiax + rk22t2 * phiaz;
      const double qke22 = qk22t1 * phiax + qk22t2 * phiaz;
      const double rke31 = rk31t1 * phiaz + rk31t2 * phiax + rk31t3 * phiaz;
      const double qke31 = qk31t1 * phiaz + qk31t2 * phiax + qk31t3 * phiaz;
      const double rke33 = rk33t1 * phiaz + rk33t2 * phiax;
      const double qke33 = qk33t1 * phiaz + qk33t2 * phiax;
      const double rke12 = rk12t1 * phiax + rk12t2 * phiax + rk12t3 * phia;
      const double qke12 = qk12t1 * phiax + qk12t2 * phiax + qk12t3 * phia;
      const double rke21 = rk21t1 * phia + rk21t2 * phia + rk21t3 * phiax;
      const double qke21 = qk21t1 * phia + qk21t2 * phia + qk21t3 * phiax;
      const double rke23 = rk23t1 * phia + rk23t2 * phia + rk23t3 * phiaz;
      const double qke23 = qk23t1 * phia + qk23t2 * phia + qk23t3 * phiaz;
      const double rke32 = rk32t1 * phiaz + rk32t2 * phiaz + rk32t3 * phia;
      const double qke32 = qk32t1 * phiaz + qk32t2 * phiaz + qk32t3 * phia;
      me0 = me0 + rme11;
      me1 = me1 + rme22;
      me2 = me2 + rme33;
      ke[0] = zadd(ke[0], dcx{rke11, qke11 + qme11});
      ke[4] = zadd(ke[4], dcx{rke22, qke22 + qme22});
      ke[8] = zadd(ke[8], dcx{rke33, qke33 + qme33});
      ke[2] = zadd(ke[2], dcx{rke13, qke13});
      ke[6] = zadd(ke[6], dcx{rke31, qke31});
      ke[1] = zsub(ke[1], dcx{-qke12, rke12});
      ke[3] = zadd(ke[3], dcx{-qke21, rke21});
      ke[5] = zadd(ke[5], dcx{-qke23, rke23});
      ke[7] = zsub(ke[7], dcx{-qke32, rke32});
    }
  out[0] = make_double2(me0 + ke[0].re, ke[0].im);
  out[1] = make_double2(0.0 + ke[1].re, ke[1].im);
  out[2] = make_double2(0.0 + ke[2].re, ke[2].im);
  out[3] = make_double2(0.0 + ke[3].re, ke[3].im);
  out[4] = make_double2(me1 + ke[4].re, ke[4].im);
  out[5] = make_double2(0.0 + ke[5].re, ke[5].im);
  out[6] = make_double2(0.0 + ke[6].re, ke[6].im);
  out[7] = make_double2(0.0 + ke[7].re, ke[7].im);
  out[8] = make_double2(me2 + ke[8].re, ke[8].im);
}

__device__ __forceinline__ dcx zneg(dcx a) { return dcx{-a.re, -a.im}; }

// CMDAMP (estiff25.f:756-961): PML version of KMDAMP, stretched derivatives
// d/dx EX, d/dz EZ, complex arithmetic in the reference's order
__device__ __forceinline__ void cmdamp_pair(const double *qc, const double *shx, const double *shz,
                                            const double *shn, int a, int b, double wpy,
                                            double2 *out) {
  const dcx cwpy = dcx{0.0, wpy}, ztwo = dcx{2.0, 0.0};
  double me0 = 0.0, me1 = 0.0, me2 = 0.0;
  dcx ce[9];
#pragma unroll
  for (int k = 0; k < 9; k++) ce[k] = dcx{0.0, 0.0};
  for (int intx = 0; intx < kNint; intx++)
    for (int intz = 0; intz < kNint; intz++) {
      const int q = intx + kNint * intz;
      const double *c = qc + kNqc * q;
      const dcx zvp2 = dcx{c[5], c[6]}, zvs2 = dcx{c[7], c[8]};
      const double rm1 = c[9], qm1 = c[10], rm2 = c[11], qm2 = c[12];
      const dcx ex = dcx{c[13], c[14]}, ez = dcx{c[15], c[16]};
      const double phib = shn[q * kNen + b];
      const dcx phibx = zmul(dcx{shx[q * kNen + b], 0.0}, ex);
      const dcx phibz = zmul(dcx{shz[q * kNen + b], 0.0}, ez);
      const dcx cphib = dcx{phib, 0.0};
      const double rm11t1 = rm1 * phib, qm11t1 = qm1 * phib;
      const double rm22t1 = rm2 * phib, qm22t1 = qm2 * phib;
      const dcx ce11t1 = zmul(zvp2, phibx), ce11t2 = zmul(zvs2, phibz);
      const dcx ce13t1 = zmul(zvp2, phibz), ce13t2 = zmul(zvs2, phibx);
      const dcx ce13t3 = zneg(zmul(zmul(ztwo, zvs2), phibz));
      const dcx ce22t1 = zmul(zvs2, phibx), ce22t2 = zmul(zvs2, phibz);
      const dcx ce31t1 = zmul(zvp2, phibx), ce31t2 = zmul(zvs2, phibz);
      const dcx ce31t3 = zneg(zmul(zmul(ztwo, zvs2), phibx));
      const dcx ce33t1 = zmul(zvp2, phibz), ce33t2 = zmul(zvs2, phibx);
      const dcx ce12t1 = zmul(zmul(cwpy, zvp2), cphib);
      const dcx ce12t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), cphib));
      const dcx ce12t3 = zneg(zmul(zmul(cwpy, zvs2), phibx));
      const dcx ce21t1 = zmul(zmul(cwpy, zvp2), phibx);
      const dcx ce21t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), phibx));
      const dcx ce21t3 = zneg(zmul(zmul(cwpy, zvs2), cphib));
      const dcx ce23t1 = zmul(zmul(cwpy, zvp2), phibz);
      const dcx ce23t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), phibz));
      const dcx ce23t3 = zneg(zmul(zmul(cwpy, zvs2), cphib));
      const dcx ce32t1 = zmul(zmul(cwpy, zvp2), cphib);
      const dcx ce32t2 = zneg(zmul(zmul(zmul(ztwo, cwpy), zvs2), cphib));
      const dcx ce32t3 = zneg(zmul(zmul(cwpy, zvs2), phibz));
      const double phia = shn[q * kNen + a];
      const dcx phiax = zmul(dcx{shx[q * kNen + a], 0.0}, ex);
      const dcx phiaz = zmul(dcx{shz[q * kNen + a], 0.0}, ez);
      const dcx cphia = dcx{phia, 0.0};
      const double rme11 = rm11t1 * phia, qme11 = qm11t1 * phia;
      const double rme22 = rm22t1 * phia, qme22 = qm22t1 * phia;
      const double rme33 = rme11, qme33 = qme11;
      const dcx ce11 = zadd(zmul(ce11t1, phiax), zmul(ce11t2, phiaz));
      const dcx ce13 = zadd(zadd(zmul(ce13t1, phiax), zmul(ce13t2, phiaz)), zmul(ce13t3, phiax));
      const dcx ce22 = zadd(zmul(ce22t1, phiax), zmul(ce22t2, phiaz));
      const dcx ce31 = zadd(zadd(zmul(ce31t1, phiaz), zmul(ce31t2, phiax)), zmul(ce31t3, phiaz));
      const dcx ce33 = zadd(zmul(ce33t1, phiaz), zmul(ce33t2, phiax));
      const dcx ce12 = zadd(zadd(zmul(ce12t1, phiax), zmul(ce12t2, phiax)), zmul(ce12t3, cphia));
      const dcx ce21 = zadd(zadd(zmul(ce21t1, cphia), zmul(ce21t2, cphia)), zmul(ce21t3, phiax));
      const dcx ce23 = zadd(zadd(zmul(ce23t1, cphia), zmul(ce23t2, cphia)), zmul(ce23t3, phiaz));
      const dcx ce32 = zadd(zadd(zmul(ce32t1, phiaz), zmul(ce32t2, phiaz)), zmul(ce32t3, cphia));
      me0 = me0 + rme11;
      me1 = me1 + rme22;
      me2 = me2 + rme33;
      ce[0] = zadd(zadd(ce[0], ce11), dcx{0.0, qme11});
      ce[1] = zsub(ce[1], ce12);
      ce[2] = zadd(ce[2], ce13);
      ce[3] = zadd(ce[3], ce21);
      ce[4] = zadd(zadd(ce[4], ce22), dcx{0.0, qme22});
      ce[5] = zadd(ce[5], ce23);
      ce[6] = zadd(ce[6], ce31);
      ce[7] = zsub(ce[7], ce32);
      ce[8] = zadd(zadd(ce[8], ce33), dcx{0.0, qme33});
    }
  out[0] = make_double2(me0 + ce[0].re, ce[0].im);
  out[1] = make_double2(0.0 + ce[1].re, ce[1].im);
  out[2] = make_double2(0.0 + ce[2].re, ce[2].im);
  out[3] = make_double2(0.0 + ce[3].re, ce[3].im);
  out[4] = make_double2(me1 + ce[4].re, ce[4].im);
  out[5] = make_double2(0.0 + ce[5].re, ce[5].im);
  out[6] = make_double2(0.0 + ce[6].re, ce[6].im);
  out[7] = make_double2(0.0 + ce[7].re, ce[7].im);
  out[8] = make_double2(me2 + ce[8].re, ce[8].im);
}

// kDisp: dispersive media (KMDAMP / CMDAMP); a separate instance so that the
// non-dispersive kernel keeps its own register allocation
template <bool kDisp>
__global__ void __launch_bounds__(kPlainThreads, 1)
    k_elem_plain(MeshView mv, DevTables dt, PlainArgs pa, double2 *__restrict__ elemmat,
                 int *__restrict__ err) {
  extern __shared__ double sm[];
  double *shx = sm + kSmShx, *shz = sm + kSmShz, *shn = sm + kSmShn, *qc = sm + kSmQ;
  const int e = pa.ebase + blockIdx.x;
  const int t = threadIdx.x;
  const int4 ie = mv.ieng[e];
  const bool pml = mv.cdomain[e] == 'A';
  // ---- per quadrature point: Jacobian, interpolated model, coefficients
  if (t < kNq) {
    const int q = t, intx = q % kNint, intz = q / kNint;
    QGeo g;
    bool ok = quad_geo(mv, dt, ie, q, pml, g);
    if (!ok) atomicCAS(err, 0, e + 1);
    double *c = qc + kNqc * q;
    c[0] = g.dxdxi; c[1] = g.dxdeta; c[2] = g.dzdxi; c[3] = g.dzdeta; c[4] = g.rjac;
    double weight = dt.wts[intx] * dt.wts[intz] * g.rjac;
    double lambda = g.lam * weight, mu = g.mu * weight, rhow = g.rho * weight;
    if constexpr (kDisp) {
      // KMDAMP / CMDAMP point terms (estiff25.f:592-607, 822-838)
      double vp, vs, qpp, qss;
      quad_qual(mv, dt, ie, q, vp, vs, qpp, qss);
      const dcx zv = vcmplx(pa, vp, qpp), zs = vcmplx(pa, vs, qss);
      dcx zvp2 = zmul(zv, zv), zvs2 = zmul(zs, zs);
      double rvp2, qvp2, rvs2, qvs2;
      if (!pml) {
        rvp2 = zvp2.re * weight;
        qvp2 = zvp2.im * weight;
        rvs2 = zvs2.re * weight;
        qvs2 = zvs2.im * weight;
      } else {
        zvp2 = zmul(zvp2, dcx{weight, 0.0});
        zvs2 = zmul(zvs2, dcx{weight, 0.0});
        rvp2 = zvp2.re;
        qvp2 = zvp2.im;
        rvs2 = zvs2.re;
        qvs2 = zvs2.im;
      }
      c[5] = rvp2; c[6] = qvp2; c[7] = rvs2; c[8] = qvs2;
      c[9] = -(pa.w2 * weight) + pa.w2 * pa.py2 * rvs2;   // RMCOEFF1
      c[10] = pa.w2 * pa.py2 * qvs2;                      // QMCOEFF1
      c[11] = -(pa.w2 * weight) + pa.w2 * pa.py2 * rvp2;  // RMCOEFF2
      c[12] = pa.w2 * pa.py2 * qvp2;                      // QMCOEFF2
      if (pml) {
        // CJCM_QUAL: the damping profile uses the interpolated Vp
        dcx ex = dcx{1.0, 0.0}, ez = dcx{1.0, 0.0};
        if (g.xdep > 2.22e-16)
          ex = zdampfn(g.xdep, vp, pa.pml.xwidth, pa.pml.dmax, pa.logr, pa.pml.kappa,
                       pa.pml.fcent, pa.omega);
        if (g.zdep > 2.22e-16)
          ez = zdampfn(g.zdep, vp, pa.pml.zwidth, pa.pml.dmax, pa.logr, pa.pml.kappa,
                       pa.pml.fcent, pa.omega);
        c[13] = ex.re; c[14] = ex.im;
        c[15] = ez.re; c[16] = ez.im;
      }
    } else if (!pml) {
      double c11 = lambda + 2.0 * mu;
      c[5] = lambda;
      c[6] = mu;
      c[7] = c11;
      c[8] = -pa.w2 * (rhow - pa.py2 * mu);   // COEFFM1 (C66)
      c[9] = -pa.w2 * (rhow - pa.py2 * c11);  // COEFFM2 (C22)
      c[10] = pa.wpy * lambda;                // WPY*C12 = WPY*C23
      c[11] = pa.wpy * mu;                    // WPY*C66 = WPY*C44
    } else {
      dcx ex = dcx{1.0, 0.0}, ez = dcx{1.0, 0.0};
      if (g.xdep > 2.22e-16)
        ex = zdampfn(g.xdep, g.vel, pa.pml.xwidth, pa.pml.dmax, pa.logr, pa.pml.kappa,
                     pa.pml.fcent, pa.omega);
      if (g.zdep > 2.22e-16)
        ez = zdampfn(g.zdep, g.vel, pa.pml.zwidth, pa.pml.dmax, pa.logr, pa.pml.kappa,
                     pa.pml.fcent, pa.omega);
      c[5] = lambda;
      c[6] = mu;
      c[7] = -pa.w2 * (rhow - pa.py2 * mu);                  // COEFFM1
      c[8] = -pa.w2 * (rhow - pa.py2 * (lambda + 2.0 * mu)); // COEFFM2
      c[9] = ex.re; c[10] = ex.im;
      c[11] = ez.re; c[12] = ez.im;
    }
  }
  __syncthreads();
  // ---- global shape-function derivatives (CJMK_TVI cjac.f:128-134)
  for (int idx = t; idx < kNq * kNen; idx += kPlainThreads) {
    const int q = idx / kNen;
    const double *c = qc + kNqc * q;
    const double *sl = dt.shl + 3 * (size_t)idx;
    double drnxi = sl[0], drneta = sl[1];
    shx[idx] = (drnxi * c[3] - drneta * c[2]) / c[4];
    shz[idx] = -(drnxi * c[1] - drneta * c[0]) / c[4];
    shn[idx] = sl[2];
  }
  __syncthreads();
  if (t >= kNab) return;
  const int a = t / kNen, b = t % kNen;
  double2 *out = elemmat + ((size_t)e * kNab + t) * 9;
  if constexpr (kDisp) {
    if (!pml)
      kmdamp_pair(qc, shx, shz, shn, a, b, pa.wpy, out);
    else
      cmdamp_pair(qc, shx, shz, shn, a, b, pa.wpy, out);
    return;
  }
  if (!pml) {
    // KM25ISOQ (estiff25.f:64-154) for the node pair (IAE=a, IBE=b)
    double me0 = 0.0, me1 = 0.0, me2 = 0.0;
    double r00 = 0.0, r02 = 0.0, r11 = 0.0, r20 = 0.0, r22 = 0.0;
    double i01 = 0.0, i10 = 0.0, i12 = 0.0, i21 = 0.0;
    for (int intx = 0; intx < kNint; intx++)
      for (int intz = 0; intz < kNint; intz++) {
        const int q = intx + kNint * intz;
        const double *c = qc + kNqc * q;
        const double lambda = c[5], mu = c[6], c11 = c[7], cm1 = c[8], cm2 = c[9];
        const double wc12 = c[10], wc66 = c[11];
        const double c13 = lambda, c33 = c11, c55 = mu, c66 = mu, c44 = mu, cm3 = cm1;
        const double phib = shn[q * kNen + b], phibx = shx[q * kNen + b], phibz = shz[q * kNen + b];
        const double phia = shn[q * kNen + a], phiax = shx[q * kNen + a], phiaz = shz[q * kNen + a];
        double phibr1 = phib * cm1, phibr2 = phib * cm2, phibr3 = phib * cm3;
        double k11t1 = c11 * phibx, k11t2 = c55 * phibz;
        double k13t1 = c13 * phibz, k13t2 = c55 * phibx;
        double k22t1 = c66 * phibx, k22t2 = c44 * phibz;
        double k31t1 = c13 * phibx, k31t2 = c55 * phibz;
        double k33t1 = c33 * phibz, k33t2 = c55 * phibx;
        double k12t1 = wc12 * phib, k12t2 = wc66 * phibx;
        double k21t1 = wc12 * phibx, k21t2 = wc66 * phib;
        double k23t1 = wc12 * phibz, k23t2 = wc66 * phib;
        double k32t1 = wc12 * phib, k32t2 = wc66 * phibz;
        me0 = me0 + phibr1 * phia;
        me1 = me1 + phibr2 * phia;
        me2 = me2 + phibr3 * phia;
        double ke11 = phiax * k11t1 + phiaz * k11t2;
        double ke13 = phiax * k13t1 + phiaz * k13t2;
        double ke22 = phiax * k22t1 + phiaz * k22t2;
        double ke31 = phiaz * k31t1 + phiax * k31t2;
        double ke33 = phiaz * k33t1 + phiax * k33t2;
        double ke12 = phiax * k12t1 - phia * k12t2;
        double ke21 = phia * k21t1 - phiax * k21t2;
        double ke23 = phia * k23t1 - phiaz * k23t2;
        double ke32 = phiaz * k32t1 - phia * k32t2;
        r00 = r00 + ke11;
        i01 = i01 - ke12;
        r02 = r02 + ke13;
        i10 = i10 + ke21;
        r11 = r11 + ke22;
        i12 = i12 + ke23;
        r20 = r20 + ke31;
        i21 = i21 - ke32;
        r22 = r22 + ke33;
      }
    // ASMBLE_CDIST: R1 = ME + Re(CE), Q1 = Im(CE)
    out[0] = make_double2(me0 + r00, 0.0);
    out[1] = make_double2(0.0 + 0.0, i01);
    out[2] = make_double2(0.0 + r02, 0.0);
    out[3] = make_double2(0.0 + 0.0, i10);
    out[4] = make_double2(me1 + r11, 0.0);
    out[5] = make_double2(0.0 + 0.0, i12);
    out[6] = make_double2(0.0 + r20, 0.0);
    out[7] = make_double2(0.0 + 0.0, i21);
    out[8] = make_double2(me2 + r22, 0.0);
  } else {
    // CM25ISOQ (estiff25.f:235-332)
    const dcx cwpy = dcx{0.0, pa.wpy};
    double me0 = 0.0, me1 = 0.0, me2 = 0.0;
    dcx ce[9];
#pragma unroll
    for (int k = 0; k < 9; k++) ce[k] = dcx{0.0, 0.0};
    for (int intx = 0; intx < kNint; intx++)
      for (int intz = 0; intz < kNint; intz++) {
        const int q = intx + kNint * intz;
        const double *c = qc + kNqc * q;
        const double lambda = c[5], mu = c[6], cm1 = c[7], cm2 = c[8], cm3 = cm1;
        const dcx ex = dcx{c[9], c[10]}, ez = dcx{c[11], c[12]};
        const dcx clam = dcx{lambda, 0.0}, cmu = dcx{mu, 0.0};
        const dcx c11 = zadd(zadd(clam, cmu), cmu), c12 = clam, c13 = clam;
        const dcx c23 = clam, c33 = zadd(zadd(clam, cmu), cmu);
        const dcx c44 = cmu, c55 = c44, c66 = c44;
        const double phib = shn[q * kNen + b];
        const dcx phibx = zmul(dcx{shx[q * kNen + b], 0.0}, ex);
        const dcx phibz = zmul(dcx{shz[q * kNen + b], 0.0}, ez);
        double phibr1 = cm1 * phib, phibr2 = cm2 * phib, phibr3 = cm3 * phib;
        dcx k11t1 = zmul(c11, phibx), k11t2 = zmul(c55, phibz);
        dcx k13t1 = zmul(c13, phibz), k13t2 = zmul(c55, phibx);
        dcx k22t1 = zmul(c66, phibx), k22t2 = zmul(c44, phibz);
        dcx k31t1 = zmul(c13, phibx), k31t2 = zmul(c55, phibz);
        dcx k33t1 = zmul(c33, phibz), k33t2 = zmul(c55, phibx);
        dcx k12t1 = zmul(zmul(cwpy, c12), dcx{phib, 0.0});
        dcx k12t2 = zmul(zmul(cwpy, c66), phibx);
        dcx k21t1 = zmul(zmul(cwpy, c12), phibx);
        dcx k21t2 = zmul(zmul(cwpy, c66), dcx{phib, 0.0});
        dcx k23t1 = zmul(zmul(cwpy, c23), phibz);
        dcx k23t2 = zmul(zmul(cwpy, c44), dcx{phib, 0.0});
        dcx k32t1 = zmul(zmul(cwpy, c23), dcx{phib, 0.0});
        dcx k32t2 = zmul(zmul(cwpy, c44), phibz);
        const double phia = shn[q * kNen + a];
        const dcx phiax = zmul(dcx{shx[q * kNen + a], 0.0}, ex);
        const dcx phiaz = zmul(dcx{shz[q * kNen + a], 0.0}, ez);
        me0 = me0 + phia * phibr1;
        me1 = me1 + phia * phibr2;
        me2 = me2 + phia * phibr3;
        dcx ce11 = zadd(zmul(phiax, k11t1), zmul(phiaz, k11t2));
        dcx ce13 = zadd(zmul(phiax, k13t1), zmul(phiaz, k13t2));
        dcx ce22 = zadd(zmul(phiax, k22t1), zmul(phiaz, k22t2));
        dcx ce31 = zadd(zmul(phiaz, k31t1), zmul(phiax, k31t2));
        dcx ce33 = zadd(zmul(phiaz, k33t1), zmul(phiax, k33t2));
        dcx ce12 = zsub(zmul(phiax, k12t1), zmul(dcx{phia, 0.0}, k12t2));
        dcx ce21 = zsub(zmul(dcx{phia, 0.0}, k21t1), zmul(phiax, k21t2));
        dcx ce23 = zsub(zmul(dcx{phia, 0.0}, k23t1), zmul(phiaz, k23t2));
        dcx ce32 = zsub(zmul(phiaz, k32t1), zmul(dcx{phia, 0.0}, k32t2));
        ce[0] = zadd(ce[0], ce11);
        ce[1] = zsub(ce[1], ce12);
        ce[2] = zadd(ce[2], ce13);
        ce[3] = zadd(ce[3], ce21);
        ce[4] = zadd(ce[4], ce22);
        ce[5] = zadd(ce[5], ce23);
        ce[6] = zadd(ce[6], ce31);
        ce[7] = zsub(ce[7], ce32);
        ce[8] = zadd(ce[8], ce33);
      }
    out[0] = make_double2(me0 + ce[0].re, ce[0].im);
    out[1] = make_double2(0.0 + ce[1].re, ce[1].im);
    out[2] = make_double2(0.0 + ce[2].re, ce[2].im);
    out[3] = make_double2(0.0 + ce[3].re, ce[3].im);
    out[4] = make_double2(me1 + ce[4].re, ce[4].im);
    out[5] = make_double2(0.0 + ce[5].re, ce[5].im);
    out[6] = make_double2(0.0 + ce[6].re, ce[6].im);
    out[7] = make_double2(0.0 + ce[7].re, ce[7].im);
    out[8] = make_double2(me2 + ce[8].re, ce[8].im);
  }
}

#ifndef FEM25_PLAIN_FMA
// Sum of the element contributions of every nonzero of [nz0, nz1) in element order:
// FP64 (complex128 output) and the reference's COMPLEX*8 accumulation
// CDIST = CDIST + CMPLX(CARG) (asmble.f90:302-305).
__global__ void k_gather_plain(long long nz0, long long nz1, const int *__restrict__ gptr,
                               const int *__restrict__ glist, const double2 *__restrict__ elemmat,
                               double2 *__restrict__ csr128, float2 *__restrict__ csr64) {
  long long nz = nz0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (nz >= nz1) return;
  double sr = 0.0, si = 0.0;
  float fr = 0.0f, fi = 0.0f;
  for (int k = gptr[nz]; k < gptr[nz + 1]; k++) {
    double2 v = elemmat[glist[k]];
    sr = sr + v.x;
    si = si + v.y;
    fr = fr + __double2float_rn(v.x);
    fi = fi + __double2float_rn(v.y);
  }
  if (csr128) csr128[nz] = make_double2(sr, si);
  if (csr64) csr64[nz] = make_float2(fr, fi);
}

// ---------------------------------------------------------------------------
// element-to-nonzero map
// ---------------------------------------------------------------------------
// ASMBLE_CDIST's lookups (IBSECT on the row, asmble.f90:295) done once.
__device__ __forceinline__ int find_col(const int *jc, int beg, int end, int col) {
  int lo = beg, hi = end - 1;  // 0-based inclusive range of jcptr
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int v = jc[mid];
    if (v == col) return mid;
    if (v < col) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// pass 0: count contributions per nonzero; pass 1: place contribution ids
__global__ void k_map_contrib(int nelem, const int *__restrict__ lm, const int *__restrict__ irptr,
                              const int *__restrict__ jcptr, int *__restrict__ count,
                              const int *__restrict__ gptr, int *__restrict__ cursor,
                              int *__restrict__ glist, int pass, int *__restrict__ err) {
  long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)nelem * kNab) return;
  int e = (int)(gid / kNab), ab = (int)(gid % kNab);
  int a = ab / kNen, b = ab % kNen;
  const int *lme = lm + (size_t)e * kNee;
  for (int i = 0; i < 3; i++) {
    int row = lme[3 * a + i];
    if (row <= 0) continue;
    int beg = irptr[row - 1] - 1, end = irptr[row] - 1;
    for (int j = 0; j < 3; j++) {
      int col = lme[3 * b + j];
      if (col <= 0) continue;
      int nz = find_col(jcptr, beg, end, col);
      if (nz < 0) {
        atomicCAS(err, 0, e + 1);
        continue;
      }
      if (pass == 0) {
        atomicAdd(&count[nz], 1);
      } else {
        int slot = atomicAdd(&cursor[nz], 1);
        glist[gptr[nz] + slot] = (int)(gid * 9 + 3 * i + j);
      }
    }
  }
}

// contributions of one nonzero come from distinct elements; order them by id
__global__ void k_sort_lists(long long n, const int *__restrict__ ptr, int *__restrict__ list,
                             int *__restrict__ err) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = ptr[i], e = ptr[i + 1];
  if (e <= b) {
    atomicCAS(err, 0, -1);
    return;
  }
  for (int k = b + 1; k < e; k++) {
    int v = list[k], m = k - 1;
    while (m >= b && list[m] > v) {
      list[m + 1] = list[m];
      m--;
    }
    list[m + 1] = v;
  }
}

__global__ void k_check_jac(MeshView mv, DevTables dt, int *__restrict__ err) {
  long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)mv.nelem * kNq) return;
  int e = (int)(gid / kNq), q = (int)(gid % kNq);
  QGeo g;
  if (!quad_geo(mv, dt, mv.ieng[e], q, mv.cdomain[e] == 'A', g)) atomicCAS(err, 0, e + 1);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
PmlParams pml_params(const Ctx *c, char cftype, double freq) {
  const fem25_mesh &m = c->mesh_scalars;
  PmlParams p;
  p.omega = 6.2831853071795862 * freq;
  bool s = (cftype == 'S');
  p.rcoeff = s ? m.rcoeff_srf : m.rcoeff_bdy;
  p.dmax = s ? m.dmax_srf : m.dmax_bdy;
  p.kappa = s ? m.kappa_srf : m.kappa_bdy;
  p.fcent = s ? m.fcent_srf : m.fcent_bdy;
  p.xwidth = m.xwidth;
  p.zwidth = m.zwidth;
  return p;
}

#endif  // FEM25_PLAIN_FMA

cudaError_t launch_elem_plain(Ctx *c, char cftype, double freq, double py, int e0, int e1,
                              cudaStream_t st) {
  if (e1 <= e0) return cudaSuccess;
  PlainArgs pa;
  pa.pml = fem25::pml_params(c, cftype, freq);
  pa.omega = pa.pml.omega;
  pa.w2 = ipow2(pa.omega);  // OMEGA**2
  pa.py2 = ipow2(py);       // PY**2
  pa.wpy = pa.omega * py;
  pa.logr = std::log(pa.pml.rcoeff);
  pa.ldisp = c->mesh_scalars.ldisp ? 1 : 0;
  pa.freq0 = c->mesh_scalars.freq0;
  pa.fac1 = (pa.ldisp && pa.freq0 != 0.0) ? std::log(freq / pa.freq0) : 0.0;
  pa.ebase = e0;
  size_t smem = sizeof(double) * kSmTot;
  if (pa.ldisp) {
    cudaError_t e = cudaFuncSetAttribute(k_elem_plain<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_elem_plain<true><<<e1 - e0, kPlainThreads, smem, st>>>(c->mv, c->dt, pa, c->d_elemmat,
                                                             c->d_err);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_elem_plain<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_elem_plain<false><<<e1 - e0, kPlainThreads, smem, st>>>(c->mv, c->dt, pa, c->d_elemmat,
                                                              c->d_err);
  }
  return cudaGetLastError();
}

#ifndef FEM25_PLAIN_FMA
cudaError_t launch_gather_plain(Ctx *c, double *csr128, float *csr64, long long nz0,
                                long long nz1, cudaStream_t st) {
  if (nz1 <= nz0) return cudaSuccess;
  int th = 256;
  long long blocks = (nz1 - nz0 + th - 1) / th;
  k_gather_plain<<<(unsigned)blocks, th, 0, st>>>(nz0, nz1, c->d_gptr, c->d_glist, c->d_elemmat,
                                                   (double2 *)csr128, (float2 *)csr64);
  return cudaGetLastError();
}

cudaError_t check_jacobians(Ctx *c, cudaStream_t st) {
  long long n = (long long)c->nelem * kNq;
  k_check_jac<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c->mv, c->dt, c->d_err);
  return cudaGetLastError();
}

// exclusive scan of int counts into ptr[0..n] (ptr[n] = total)
cudaError_t scan_counts(const int *count, int *ptr, long long n, cudaStream_t st) {
  size_t tmp = 0;
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tmp, count, ptr, (int)(n + 1), st);
  if (e != cudaSuccess) return e;
  void *d_tmp = nullptr;
  e = cudaMallocAsync(&d_tmp, tmp, st);
  if (e != cudaSuccess) return e;
  e = cub::DeviceScan::ExclusiveSum(d_tmp, tmp, count, ptr, (int)(n + 1), st);
  cudaFreeAsync(d_tmp, st);
  return e;
}

cudaError_t build_gather_map(Ctx *c, cudaStream_t st) {
  cudaError_t e;
  int *d_count = nullptr, *d_cursor = nullptr;
  long long n = c->nzero;
  if ((e = cudaMallocAsync(&d_count, sizeof(int) * (n + 1), st))) return e;
  if ((e = cudaMallocAsync(&d_cursor, sizeof(int) * (n + 1), st))) return e;
  cudaMemsetAsync(d_count, 0, sizeof(int) * (n + 1), st);
  cudaMemsetAsync(d_cursor, 0, sizeof(int) * (n + 1), st);
  if ((e = cudaMalloc(&c->d_gptr, sizeof(int) * (n + 1)))) return e;
  long long tot = (long long)c->nelem * kNab;
  unsigned nb = (unsigned)((tot + 255) / 256);
  k_map_contrib<<<nb, 256, 0, st>>>(c->nelem, c->d_lm, c->d_irptr, c->d_jcptr, d_count, nullptr,
                                     nullptr, nullptr, 0, c->d_err);
  if ((e = scan_counts(d_count, c->d_gptr, n, st))) return e;
  int total = 0;
  cudaMemcpyAsync(&total, c->d_gptr + n, sizeof(int), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st))) return e;
  c->ncontrib = total;
  if ((e = cudaMalloc(&c->d_glist, sizeof(int) * (size_t)(total > 0 ? total : 1)))) return e;
  k_map_contrib<<<nb, 256, 0, st>>>(c->nelem, c->d_lm, c->d_irptr, c->d_jcptr, nullptr, c->d_gptr,
                                     d_cursor, c->d_glist, 1, c->d_err);
  k_sort_lists<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, c->d_gptr, c->d_glist, c->d_err);
  cudaFreeAsync(d_count, st);
  cudaFreeAsync(d_cursor, st);
  return cudaGetLastError();
}

#endif  // FEM25_PLAIN_FMA

#ifdef FEM25_PLAIN_FMA
}  // namespace plain_fma

cudaError_t launch_elem_plain_fma(Ctx *c, char cftype, double freq, double py, int e0, int e1,
                                  cudaStream_t st) {
  return plain_fma::launch_elem_plain(c, cftype, freq, py, e0, e1, st);
}
#endif
}  // namespace fem25
