// Kernels that reproduce the reference's single-precision bookkeeping around
// the operator: the Bielak effective force ASMB_PEFF (asmble.f90:318-377),
// the forward misfit / adjoint source (EXRESP25D, CRESID, BPRESID4, COBJ4,
// RESID_DRHS) and the reference-compatible virtual-force gradient
// (CFMAT_DIST / VFORCE25 / DJACAB / DKM_VPVS, ADJFLAM_DIST).
//
// Compiled with -fmad=false so every COMPLEX*8 / REAL*8 operation is rounded
// on its own, as the reference writes it.
#include <algorithm>

#include <complex>

#include "ctx.cuh"
#include "kcommon.cuh"

namespace fem25 {

// ---------------------------------------------------------------------------
// ASMB_PEFF: PEFF(i) -= S_ij ue_j for (B,E) pairs, += for (E,B) pairs
// ---------------------------------------------------------------------------
__global__ void k_peff(int ndof, int nsrc, const int *__restrict__ irptr, const int *__restrict__ jcptr,
                       const char *__restrict__ cnp, const float2 *__restrict__ a,
                       const float2 *__restrict__ ue, float2 *__restrict__ peff) {
  long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)ndof * nsrc) return;
  const int s = (int)(gid / ndof), row = (int)(gid % ndof);  // row 0-based
  const float2 *u = ue + (size_t)s * ndof;
  float br = 0.0f, bi = 0.0f;
  const char c1 = cnp[row];
  if (c1 == 'B' || c1 == 'E') {
    for (int j = irptr[row] - 1; j < irptr[row + 1] - 1; j++) {
      const int col = jcptr[j] - 1;
      const char c2 = cnp[col];
      const float2 av = a[j], uv = u[col];
      const float pr = av.x * uv.x - av.y * uv.y, pi = av.x * uv.y + av.y * uv.x;
      if (c1 == 'B' && c2 == 'E') {
        br = br - pr;
        bi = bi - pi;
      } else if (c1 == 'E' && c2 == 'B') {
        br = br + pr;
        bi = bi + pi;
      }
    }
  }
  peff[gid] = make_float2(br, bi);
}

cudaError_t launch_peff(Ctx *c, int nsrc, const float *a_loc, const float *ue, float *peff,
                        cudaStream_t st) {
  long long n = (long long)c->ndof * nsrc;
  k_peff<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c->ndof, nsrc, c->d_irptr, c->d_jcptr,
                                                      c->d_cnp, (const float2 *)a_loc,
                                                      (const float2 *)ue, (float2 *)peff);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// ADDBLK (bielak_utils.f:1116-1125): SOL(i) += U0(i) on the 'E' DOFs, for
// nsrc solutions at once
// ---------------------------------------------------------------------------
__global__ void k_addblk(int ndof, int nsrc, const char *__restrict__ cnp,
                         const float2 *__restrict__ u0, float2 *__restrict__ sol) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)ndof * nsrc) return;
  if (cnp[gid % ndof] != 'E') return;
  const float2 a = sol[gid], b = u0[gid];
  sol[gid] = make_float2(a.x + b.x, a.y + b.y);
}

cudaError_t launch_addblk(Ctx *c, int nsrc, const float *u0, float *sol, cudaStream_t st) {
  const long long n = (long long)c->ndof * nsrc;
  k_addblk<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(c->ndof, nsrc, c->d_cnp,
                                                        (const float2 *)u0, (float2 *)sol);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// misfit + adjoint source, one thread per (source, receiver)
//   trig[ir] = (cos, sin) of omega*py*yrec in single precision; rot = (cos th,
//   sin th, cos -th, sin -th) of the model azimuth (computed on the host).
//   The COBJ4 term (objfn.f:60-125) and the BPRESID4 residual
//   (objfn.f:795-843) follow the context's misfit options (NORM, IRESTP,
//   DTMAX, COBJ4's EPS / THRESH); the residual is scaled by HDIFFER
//   (adjgrad.f90:528-566, evaluated on the host) in RESID_DRHS.
//   |z| = sqrt(re^2 + im^2); complex products (ac - bd, ad + bc); this unit
//   is compiled without FMA contraction, so every result is bit-identical to
//   the oracle except where IRESTP = 1 or a DTMAX test takes phases
//   (atan2f, cosf, sinf of the device against the host's libm).
// ---------------------------------------------------------------------------
struct cfl {
  float re, im;
};
__device__ __forceinline__ cfl cmulf(cfl a, cfl b) {
  return cfl{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ float cabsf_(cfl z) { return sqrtf(z.re * z.re + z.im * z.im); }

// CRESID (objfn.f:953-1010)
__device__ __forceinline__ cfl cresid(int irestp, cfl obs, cfl est) {
  if (obs.re == 0.0f && obs.im == 0.0f) return cfl{0.0f, 0.0f};
  if (irestp == 1 || irestp == 2) {
    float adata, pdata, aest, pest;
    if (irestp == 2) {
      adata = sqrtf(obs.re * obs.re + obs.im * obs.im);
      pdata = 0.0f;
      aest = sqrtf(est.re * est.re + est.im * est.im);
      pest = 0.0f;
    } else {
      adata = 1.0f;
      pdata = atan2f(obs.im, obs.re);
      aest = 1.0f;
      pest = atan2f(est.im, est.re);
    }
    const cfl a = cmulf(cfl{adata, 0.0f}, cfl{cosf(pdata), sinf(pdata)});
    const cfl b = cmulf(cfl{aest, 0.0f}, cfl{cosf(pest), sinf(pest)});
    return cfl{a.re - b.re, a.im - b.im};
  }
  return cfl{obs.re - est.re, obs.im - est.im};
}

// the wrapped phase difference SPHASE(obs) - SPHASE(est) exceeds dtmax as a
// time shift (objfn.f:106-112, :826-832)
__device__ __forceinline__ bool phase_jump(cfl obs, cfl est, double freq, float dtmax) {
  const float kTwoPi = 6.283185307179586f, kPi = 3.1415926535897931f;
  float dphi = atan2f(obs.im, obs.re) - atan2f(est.im, est.re);
  if (dphi < -kPi) dphi = dphi + kTwoPi;
  if (dphi > +kPi) dphi = dphi - kTwoPi;
  return fabs((double)dphi / ((double)kTwoPi * freq)) > (double)dtmax;
}

// Receiver ir of source s: the estimates, the three COBJ4 terms (part[0..2])
// and the right-hand-side entries at its DOFs; sv[i] is the solution at
// MRDOF(i, ir) (unused where MRDOF is 0).
__device__ __forceinline__ void misfit_one(int s, int ir, int nrec, int ndof,
                                           const int *__restrict__ mrdof, const float4 tg,
                                           float4 rot, const float2 *__restrict__ recv,
                                           const float2 *sv, const float2 *__restrict__ obs,
                                           const float *__restrict__ wghts, const MisfitOpts &mo,
                                           float2 *__restrict__ est, float2 *__restrict__ rhs,
                                           float *part) {
  const cfl cf = cfl{tg.x, tg.y}, cf2 = cfl{tg.z, tg.w};
  cfl e3[3], o3[3];
  for (int i = 0; i < 3; i++) {
    int d = mrdof[3 * ir + i];
    if (d != 0) {
      float2 rv = recv[3 * ir + i];
      e3[i] = cmulf(cmulf(cfl{rv.x, rv.y}, cfl{sv[i].x, sv[i].y}), cf);
    } else {
      e3[i] = cfl{0.0f, 0.0f};
    }
    est[((size_t)s * nrec + ir) * 3 + i] = make_float2(e3[i].re, e3[i].im);
    float2 ov = obs[((size_t)s * nrec + ir) * 3 + i];
    o3[i] = cfl{ov.x, ov.y};
  }
  const float ct = rot.x, st = rot.y;
  cfl er[3];
  er[0] = cfl{e3[0].re * ct - e3[1].re * st, e3[0].im * ct - e3[1].im * st};
  er[1] = cfl{e3[0].re * st + e3[1].re * ct, e3[0].im * st + e3[1].im * ct};
  er[2] = e3[2];
  cfl res[3];
  for (int i = 0; i < 3; i++) {
    res[i] = cfl{0.0f, 0.0f};
    part[i] = 0.0f;
    if (o3[i].re == 0.0f && o3[i].im == 0.0f) continue;
    const float w = wghts[((size_t)s * nrec + ir) * 3 + i];
    const cfl S = cfl{w, 0.0f};
    const float sabs = fabsf(w);
    // ---- COBJ4 term on the unshifted pair
    {
      const cfl dif = cresid(mo.irestp, o3[i], er[i]);
      float c;
      if (mo.norm == 1) {
        c = cabsf_(cmulf(S, dif));
      } else if (mo.norm == 3) {
        const float arg = cabsf_(cmulf(S, dif));
        c = arg <= mo.eps ? arg * arg / (2.0f * mo.eps) : arg - mo.eps / 2.0f;
      } else if (mo.norm == 4) {
        const float arg = cabsf_(dif), sd = cabsf_(cmulf(S, dif));
        c = arg <= mo.thresh ? sd * sd / (2.0f * (mo.eps * mo.eps)) : sd / mo.eps;
      } else {
        const cfl cd = cmulf(cfl{dif.re, -dif.im}, dif);
        c = sabs * sabs * cd.re;
        if (mo.dtmax_obj > 0.0f && phase_jump(o3[i], er[i], mo.freq, mo.dtmax_obj)) {
          const float damp = cabsf_(o3[i]) - cabsf_(er[i]);
          c = mo.irestp == 1 ? sabs * sabs * 4.0f : sabs * sabs * (damp * damp);
        }
      }
      part[i] = c;
    }
    // ---- BPRESID4 residual on the shifted pair (EPS = 0, objfn.f:795-797)
    {
      const cfl ob = cmulf(o3[i], cf2), es = cmulf(er[i], cf2);
      const cfl dif = cresid(mo.irestp, ob, es);
      const float e0 = 0.0f;
      if (mo.norm == 1 || (mo.norm == 3 && !(cabsf_(cmulf(S, dif)) <= e0))) {
        const cfl num = cmulf(S, dif);  // CONJG(WEIGHT) = WEIGHT
        const float den = cabsf_(dif);
        res[i] = cfl{num.re / den, num.im / den};
      } else if (mo.norm == 3) {
        res[i] = cmulf(cfl{sabs * sabs / e0, 0.0f}, dif);
      } else if (mo.norm == 4) {
        const float eps2 = 0.0f;  // EPSS * EPS**2 with EPS = 0
        const float sd = cabsf_(cmulf(S, dif));
        const float denon = eps2 * sqrtf(1.0f + sd * sd / eps2);
        res[i] = cmulf(cfl{sabs * sabs / denon, 0.0f}, dif);
      } else {
        res[i] = cmulf(cfl{sabs * sabs, 0.0f}, dif);
        if (mo.dtmax > 0.0f && phase_jump(ob, es, mo.freq, mo.dtmax)) res[i] = cfl{0.0f, 0.0f};
      }
    }
  }
  const float ct2 = rot.z, st2 = rot.w;
  cfl rr[3];
  rr[0] = cfl{res[0].re * ct2 - res[1].re * st2, res[0].im * ct2 - res[1].im * st2};
  rr[1] = cfl{res[0].re * st2 + res[1].re * ct2, res[0].im * st2 + res[1].im * ct2};
  rr[2] = res[2];
  const cfl hf = cfl{mo.hfact.x, mo.hfact.y};
  for (int i = 0; i < 3; i++) {
    int d = mrdof[3 * ir + i];
    if (d <= 0 || d > ndof) continue;
    // receivers map to distinct DOFs (checked by the host): RHS = 0 + HFACT
    // RESID, conjugated for the transpose solve (adjgrad.f90:509-521)
    const cfl t = cmulf(hf, rr[i]);
    rhs[(size_t)s * ndof + d - 1] = make_float2(0.0f + t.re, -(0.0f + t.im));
  }
}

__global__ void k_misfit(int nsrc, int nrec, int ndof, const int *__restrict__ mrdof,
                         const float4 *__restrict__ trig, float4 rot, const float2 *__restrict__ recv,
                         const float2 *__restrict__ sol, const float2 *__restrict__ obs,
                         const float *__restrict__ wghts, MisfitOpts mo, float2 *__restrict__ est,
                         float2 *__restrict__ rhs, float *__restrict__ part) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nsrc * nrec) return;
  const int s = gid / nrec, ir = gid % nrec;
  float2 sv[3];
  for (int i = 0; i < 3; i++) {
    const int d = mrdof[3 * ir + i];
    sv[i] = d != 0 ? sol[(size_t)s * ndof + d - 1] : make_float2(0.0f, 0.0f);
  }
  misfit_one(s, ir, nrec, ndof, mrdof, trig[ir], rot, recv, sv, obs, wghts, mo, est, rhs,
             part + (size_t)gid * 3);
}

// RESID_DRHS conjugates the whole right-hand side (adjgrad.f90:519-521): the
// untouched entries become (0, -0)
__global__ void k_fill_conj_zero(long long n, float2 *__restrict__ rhs) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rhs[i] = make_float2(0.0f, -0.0f);
}

// per-source sum of the receiver partials in receiver order (COBJ4 order)
__global__ void k_misfit_sum(int nsrc, int nrec, const float *__restrict__ part,
                             float *__restrict__ out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsrc) return;
  // COBJ4 order: receivers, then components, skipping absent observations
  float acc = 0.0f;
  for (int k = 0; k < 3 * nrec; k++) {
    float v = part[(size_t)s * nrec * 3 + k];
    if (v != 0.0f) acc = acc + v;
  }
  out[s] = acc;
}

// The call's options: the context's, with FREQ and HDIFFER (adjgrad.f90:528-566)
// evaluated on the host (REAL*4 OMEGA, the C library's complex square root).
static MisfitOpts misfit_opts(const Ctx *c, double freq) {
  MisfitOpts mo = c->mopt;
  mo.freq = freq;
  const float omega = (float)(2.0 * 3.1415926535897932384626434 * freq);
  std::complex<float> h(1.0f, 0.0f);
  if (mo.ibphase == 1 || mo.ibphase == 2) {
    h = std::sqrt(std::complex<float>(0.0f, -omega));
    if (mo.ibphase == 2) h = -h;
  } else if (mo.ibphase == 3 || mo.ibphase == 4) {
    h = std::sqrt(std::complex<float>(0.0f, omega));
    if (mo.ibphase == 4) h = -h;
  } else if (mo.ibphase == 5) {
    h = std::complex<float>(0.0f, omega);
  } else if (mo.ibphase == 6) {
    h = std::complex<float>(0.0f, 1.0f);
  }
  mo.hfact = make_float2(h.real(), h.imag());
  return mo;
}

cudaError_t launch_misfit(Ctx *c, int nsrc, int nrec, const int *d_mrdof, const float *d_trig,
                          double freq, double py, double azmod, const float *d_recv,
                          const float *sol, const float *d_obs, const float *d_wghts,
                          float *d_est, float *rhs, float *d_misfit, cudaStream_t st) {
  (void)py;
  const MisfitOpts mo = misfit_opts(c, freq);
  float th = (float)azmod * 0.017453292519943295f;
  float4 rot = make_float4(cosf(th), sinf(th), cosf(-th), sinf(-th));
  float *d_part = nullptr;
  cudaError_t e = cudaMallocAsync(&d_part, sizeof(float) * 3 * (size_t)nsrc * nrec, st);
  if (e) return e;
  const long long nrhs = (long long)nsrc * c->ndof;
  k_fill_conj_zero<<<(unsigned)((nrhs + 255) / 256), 256, 0, st>>>(nrhs, (float2 *)rhs);
  int n = nsrc * nrec;
  k_misfit<<<(n + 127) / 128, 128, 0, st>>>(nsrc, nrec, c->ndof, d_mrdof, (const float4 *)d_trig,
                                            rot, (const float2 *)d_recv, (const float2 *)sol,
                                            (const float2 *)d_obs, d_wghts, mo, (float2 *)d_est,
                                            (float2 *)rhs, d_part);
  k_misfit_sum<<<(nsrc + 127) / 128, 128, 0, st>>>(nsrc, nrec, d_part, d_misfit);
  cudaFreeAsync(d_part, st);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// the pass after the solve, fused (one launch for all sources of a group):
// ADDBLK (bielak_utils.f:1116-1125) on the exterior DOFs, EXRESP25D
// receiver extraction (locrec2d.f:867-925) and the misfit / adjoint source
// of k_misfit.  Block s < nsrc first handles the receivers of source s: each
// thread adds the background field to its receiver DOFs itself (the same
// FP32 add as ADDBLK), computes the receiver's terms with misfit_one into
// shared memory, and thread 0 sums them in COBJ4 order.  Then every block
// takes a grid-strided share of the [nsrc][NDOF] entries that are not
// receiver DOFs (rbits): ADDBLK on 'E' DOFs, RESID_DRHS's conjugated zero in
// the right-hand side.  Receiver DOFs are distinct, so no entry has two
// writers; the results equal fem25_addblk_dev followed by fem25_misfit_dev
// bit for bit.
// ---------------------------------------------------------------------------
__global__ void k_postsolve(int nsrc, int nrec, int ndof, const char *__restrict__ cnp,
                            const uint32_t *__restrict__ rbits, const int *__restrict__ mrdof,
                            const float4 *__restrict__ trig, float4 rot,
                            const float2 *__restrict__ recv, const float2 *__restrict__ ue,
                            float2 *__restrict__ sol, const float2 *__restrict__ obs,
                            const float *__restrict__ wghts, MisfitOpts mo,
                            float2 *__restrict__ est, float2 *__restrict__ rhs,
                            float *__restrict__ misfit) {
  extern __shared__ float ps[];  // [3 nrec] COBJ4 terms of this block's source
  const int s = blockIdx.x;
  if (s < nsrc) {
    for (int ir = threadIdx.x; ir < nrec; ir += blockDim.x) {
      float2 sv[3];
      for (int i = 0; i < 3; i++) {
        const int d = mrdof[3 * ir + i];
        sv[i] = make_float2(0.0f, 0.0f);
        if (d <= 0) continue;
        const size_t k = (size_t)s * ndof + d - 1;
        float2 v = sol[k];
        if (cnp[d - 1] == 'E') {
          const float2 b = ue[k];
          v = make_float2(v.x + b.x, v.y + b.y);
          sol[k] = v;
        }
        sv[i] = v;
      }
      misfit_one(s, ir, nrec, ndof, mrdof, trig[ir], rot, recv, sv, obs, wghts, mo, est, rhs,
                 ps + 3 * ir);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      float acc = 0.0f;
      for (int k = 0; k < 3 * nrec; k++) {
        const float v = ps[k];
        if (v != 0.0f) acc = acc + v;
      }
      misfit[s] = acc;
    }
  }
  const long long n = (long long)nsrc * ndof;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int d = (int)(idx % ndof);
    if ((rbits[d >> 5] >> (d & 31)) & 1u) continue;
    if (cnp[d] == 'E') {
      const float2 a = sol[idx], b = ue[idx];
      sol[idx] = make_float2(a.x + b.x, a.y + b.y);
    }
    rhs[idx] = make_float2(0.0f, -0.0f);
  }
}

cudaError_t launch_postsolve(Ctx *c, int nsrc, int nrec, const int *d_mrdof, const uint32_t *d_bits,
                             const float *d_trig, double freq, double azmod, const float *d_recv,
                             const float *ue, float *sol, const float *d_obs, const float *d_wghts,
                             float *d_est, float *rhs, float *d_misfit, cudaStream_t st) {
  const MisfitOpts mo = misfit_opts(c, freq);
  float th = (float)azmod * 0.017453292519943295f;
  float4 rot = make_float4(cosf(th), sinf(th), cosf(-th), sinf(-th));
  const size_t smem = sizeof(float) * 3 * (size_t)nrec;
  cudaError_t e = cudaFuncSetAttribute(k_postsolve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)std::max(smem, (size_t)1));
  if (e != cudaSuccess) return e;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const long long n = (long long)nsrc * c->ndof;
  const int grid = (int)std::max<long long>(nsrc, std::min<long long>(8LL * nsm, (n + 255) / 256));
  k_postsolve<<<grid, 256, smem, st>>>(nsrc, nrec, c->ndof, c->d_cnp, d_bits, d_mrdof,
                                       (const float4 *)d_trig, rot, (const float2 *)d_recv,
                                       (const float2 *)ue, (float2 *)sol, (const float2 *)d_obs,
                                       d_wghts, mo, (float2 *)d_est, (float2 *)rhs, d_misfit);
  return cudaGetLastError();
}

// The same three launches with the per-(source, receiver) partials in a
// caller-provided device buffer of 3 * nsrc * nrec floats (every entry is
// written by k_misfit before k_misfit_sum reads it).
cudaError_t launch_misfit_part(Ctx *c, int nsrc, int nrec, const int *d_mrdof, const float *d_trig,
                               double freq, double azmod, const float *d_recv, const float *sol,
                               const float *d_obs, const float *d_wghts, float *d_est, float *rhs,
                               float *d_part, float *d_misfit, cudaStream_t st) {
  const MisfitOpts mo = misfit_opts(c, freq);
  float th = (float)azmod * 0.017453292519943295f;
  float4 rot = make_float4(cosf(th), sinf(th), cosf(-th), sinf(-th));
  const long long nrhs = (long long)nsrc * c->ndof;
  k_fill_conj_zero<<<(unsigned)((nrhs + 255) / 256), 256, 0, st>>>(nrhs, (float2 *)rhs);
  int n = nsrc * nrec;
  k_misfit<<<(n + 127) / 128, 128, 0, st>>>(nsrc, nrec, c->ndof, d_mrdof, (const float4 *)d_trig,
                                            rot, (const float2 *)d_recv, (const float2 *)sol,
                                            (const float2 *)d_obs, d_wghts, mo, (float2 *)d_est,
                                            (float2 *)rhs, d_part);
  k_misfit_sum<<<(nsrc + 127) / 128, 128, 0, st>>>(nsrc, nrec, d_part, d_misfit);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// reference-compatible virtual forces: one CTA per CSC column (inversion
// anchor), elements of MCONN in order.  DKM_VPVS (dstiff25.f:498-662) is
// evaluated by 625 threads (node pairs) into shared memory as COMPLEX*8
// CARG = CMPLX(DCMPLX(DME) + DKE) (vforce25.f:311-312), then 75 threads form
// FORCEV(row) += CARG * WAVE * CWGHT in IQE order (vforce25.f:326-330).
// ---------------------------------------------------------------------------
constexpr int kRefThreads = 640;

struct RefArgs {
  double omega, py, vpvs2;
  int lisp, accumulate, ncon, nnpg;
};

__global__ void __launch_bounds__(kRefThreads, 1)
    k_ref_cfmat(MeshView mv, DevTables dt, RefArgs ra, const int *__restrict__ lm,
                const int *__restrict__ anchor_of_col, const int *__restrict__ mconn,
                const double *__restrict__ elem_wts, const int *__restrict__ jcsc,
                const int *__restrict__ icsc, const float2 *__restrict__ wave,
                float2 *__restrict__ fmat, int *__restrict__ err) {
  extern __shared__ double sm[];
  double *shx = sm, *shz = sm + kNq * kNen, *shn = sm + 2 * kNq * kNen;
  double *qc = sm + 3 * kNq * kNen;                       // [kNq][8]
  float2 *carg = reinterpret_cast<float2 *>(qc + 8 * kNq); // [75][75]
  const int col = blockIdx.x, t = threadIdx.x;
  const int p = anchor_of_col[col];  // 0-based anchor (INPG-1)
  const int i1 = jcsc[col] - 1, i2 = jcsc[col + 1] - 1, nnzrow = i2 - i1;
  float2 *forcev = fmat + i1;
  for (int k = t; k < nnzrow; k += kRefThreads) forcev[k] = make_float2(0.0f, 0.0f);
  // elements of the anchor, in MCONN order; without accumulation only the
  // last one leaves a trace in FORCEV
  int elist[8], ne = 0;
  for (int ic = 0; ic < ra.ncon && ic < 8; ic++) {
    int e = mconn[p + (size_t)ra.nnpg * ic];
    if (e <= 0) break;
    elist[ne++] = e - 1;
  }
  const int first = ra.accumulate ? 0 : (ne > 0 ? ne - 1 : 0);
  const double wpy = ra.omega * ra.py, py2 = ipow2(ra.py), w2 = ipow2(ra.omega);
  __syncthreads();
  for (int ie_ = first; ie_ < ne; ie_++) {
    const int e = elist[ie_];
    const int4 ie = mv.ieng[e];
    if (t < kNq) {
      const int q = t, intx = q % kNint, intz = q / kNint;
      QGeo g;
      if (!quad_geo(mv, dt, ie, q, false, g)) atomicCAS(err, 0, e + 1);
      // DJACAB (djac.f:90-110): DAB = sum_ia 2 alpha_ia SF(ia), alpha nonzero
      // only at the collocated anchor
      const int il[4] = {ie.x - 1, ie.y - 1, ie.z - 1, ie.w - 1};
      double dab1 = 0.0, dab2 = 0.0;
      for (int ia = 0; ia < 4; ia++) {
        double alpha = 0.0, beta = 0.0;
        if (il[ia] == p) {
          alpha = sqrt((mv.lam[p] + 2.0 * mv.mu[p]) / mv.rho[p]);
          beta = sqrt(mv.mu[p] / mv.rho[p]);
        }
        dab1 = dab1 + 2.0 * alpha * dt.sf[4 * q + ia];
        dab2 = dab2 + 2.0 * beta * dt.sf[4 * q + ia];
      }
      double dvp, dvs;
      if (ra.lisp) {
        dvp = dab1;
        dvs = dab1 / ra.vpvs2;
      } else {
        dvp = dab2 * ra.vpvs2;
        dvs = dab2;
      }
      double *c = qc + 8 * q;
      c[0] = g.dxdxi; c[1] = g.dxdeta; c[2] = g.dzdxi; c[3] = g.dzdeta; c[4] = g.rjac;
      double weight = dt.wts[intx] * dt.wts[intz] * g.rjac;
      c[5] = dvp * weight;  // DRVP
      c[6] = dvs * weight;  // DRVS
    }
    __syncthreads();
    for (int idx = t; idx < kNq * kNen; idx += kRefThreads) {
      const int q = idx / kNen;
      const double *c = qc + 8 * q;
      const double *sl = dt.shl + 3 * (size_t)idx;
      double drnxi = sl[0], drneta = sl[1];
      shx[idx] = (drnxi * c[3] - drneta * c[2]) / c[4];
      shz[idx] = -(drnxi * c[1] - drneta * c[0]) / c[4];
      shn[idx] = sl[2];
    }
    __syncthreads();
    if (t < kNab) {
      const int a = t / kNen, b = t % kNen;
      double m0 = 0.0, m1 = 0.0, m2 = 0.0;
      double r00 = 0.0, r11 = 0.0, r22 = 0.0, r02 = 0.0, r20 = 0.0;
      double r01 = 0.0, r10 = 0.0, r12 = 0.0, r21 = 0.0;
      for (int intx = 0; intx < kNint; intx++)
        for (int intz = 0; intz < kNint; intz++) {
          const int q = intx + kNint * intz;
          const double drvp = qc[8 * q + 5], drvs = qc[8 * q + 6];
          const double rm1 = w2 * py2 * drvs, rm2 = w2 * py2 * drvp;
          const double phib = shn[q * kNen + b], phibx = shx[q * kNen + b], phibz = shz[q * kNen + b];
          const double phia = shn[q * kNen + a], phiax = shx[q * kNen + a], phiaz = shz[q * kNen + a];
          double rm11t1 = rm1 * phib, rm22t1 = rm2 * phib;
          double rk11t1 = drvp * phibx, rk11t2 = drvs * phibz;
          double rk13t1 = drvp * phibz, rk13t2 = drvs * phibx, rk13t3 = -2.0 * drvs * phibz;
          double rk22t1 = drvs * phibx, rk22t2 = drvs * phibz;
          double rk31t1 = drvp * phibx, rk31t2 = drvs * phibz, rk31t3 = -2.0 * drvs * phibx;
          double rk33t1 = drvp * phibz, rk33t2 = drvs * phibx;
          double rk12t1 = wpy * drvp * phib, rk12t2 = -2.0 * wpy * drvs * phib, rk12t3 = -wpy * drvs * phibx;
          double rk21t1 = wpy * drvp * phibx, rk21t2 = -2.0 * wpy * drvs * phibx, rk21t3 = -wpy * drvs * phib;
          double rk23t1 = wpy * drvp * phibz, rk23t2 = -2.0 * wpy * drvs * phibz, rk23t3 = -wpy * drvs * phib;
          double rk32t1 = wpy * drvp * phib, rk32t2 = -2.0 * wpy * drvs * phib, rk32t3 = -wpy * drvs * phibz;
          double rme11 = rm11t1 * phia, rme22 = rm22t1 * phia, rme33 = rme11;
          m0 = m0 + rme11;
          m1 = m1 + rme22;
          m2 = m2 + rme33;
          r00 = r00 + (rk11t1 * phiax + rk11t2 * phiaz);
          r11 = r11 + (rk22t1 * phiax + rk22t2 * phiaz);
          r22 = r22 + (rk33t1 * phiaz + rk33t2 * phiax);
          r02 = r02 + (rk13t1 * phiax + rk13t2 * phiaz + rk13t3 * phiax);
          r20 = r20 + (rk31t1 * phiaz + rk31t2 * phiax + rk31t3 * phiaz);
          r01 = r01 - (rk12t1 * phiax + rk12t2 * phiax + rk12t3 * phia);
          r10 = r10 + (rk21t1 * phia + rk21t2 * phia + rk21t3 * phiax);
          r12 = r12 + (rk23t1 * phia + rk23t2 * phia + rk23t3 * phiaz);
          r21 = r21 - (rk32t1 * phiaz + rk32t2 * phiaz + rk32t3 * phia);
        }
      // CARG = CMPLX(DCMPLX(DME,0) + DKE): DKE is real in every entry
      const int ipe = 3 * a, iqe = 3 * b;
      float2 *row0 = carg + (size_t)ipe * kNee + iqe;
      row0[0] = make_float2(__double2float_rn(m0 + r00), __double2float_rn(0.0 + 0.0));
      row0[1] = make_float2(__double2float_rn(0.0 + r01), __double2float_rn(0.0 + 0.0));
      row0[2] = make_float2(__double2float_rn(0.0 + r02), __double2float_rn(0.0 + 0.0));
      float2 *row1 = row0 + kNee;
      row1[0] = make_float2(__double2float_rn(0.0 + r10), __double2float_rn(0.0 + 0.0));
      row1[1] = make_float2(__double2float_rn(m1 + r11), __double2float_rn(0.0 + 0.0));
      row1[2] = make_float2(__double2float_rn(0.0 + r12), __double2float_rn(0.0 + 0.0));
      float2 *row2 = row1 + kNee;
      row2[0] = make_float2(__double2float_rn(0.0 + r20), __double2float_rn(0.0 + 0.0));
      row2[1] = make_float2(__double2float_rn(0.0 + r21), __double2float_rn(0.0 + 0.0));
      row2[2] = make_float2(__double2float_rn(m2 + r22), __double2float_rn(0.0 + 0.0));
    }
    __syncthreads();
    if (!ra.accumulate)
      for (int k = t; k < nnzrow; k += kRefThreads) forcev[k] = make_float2(0.0f, 0.0f);
    __syncthreads();
    if (t < kNee) {
      const int ipe = t;
      const int *lme = lm + (size_t)e * kNee;
      const int idof = lme[ipe];
      if (idof > 0) {
        // IBSECT on the CSC column
        int lo = 0, hi = nnzrow - 1, inz = -1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1, v = icsc[i1 + mid];
          if (v == idof) { inz = mid; break; }
          if (v < idof) lo = mid + 1;
          else hi = mid - 1;
        }
        if (inz < 0) {
          atomicCAS(err, 0, -(col + 1));
        } else {
          const float cw = __double2float_rn(elem_wts[e]);
          float fr = forcev[inz].x, fi = forcev[inz].y;
          for (int iqe = 0; iqe < kNee; iqe++) {
            const int jdof = lme[iqe];
            if (jdof <= 0) continue;
            const float2 cv = carg[(size_t)ipe * kNee + iqe], wv = wave[jdof - 1];
            cfl t1 = cmulf(cfl{cv.x, cv.y}, cfl{wv.x, wv.y});
            cfl t2 = cmulf(t1, cfl{cw, 0.0f});
            fr = fr + t2.re;
            fi = fi + t2.im;
          }
          forcev[inz] = make_float2(fr, fi);
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// VFORCE25_2 (vforce25.f:373-607) with DABMKISOB25 (dstiff25.f:1-203): one CTA
// per CSC column (inversion anchor); the connected elements of MCONN in
// order, no element weights, no reset between elements.  For each element
// 625 threads (node pairs) integrate the alpha and/or beta derivative blocks
// into shared memory as COMPLEX*8 CARG = CMPLX(DCMPLX(DMD,0) + DKD), then 75
// threads add CARG * WAVE to their row of each variable's force column.
// fmat: [nvar][nz] (alpha first).
// ---------------------------------------------------------------------------
struct VfArgs {
  double omega, py;
  int lisp, liss, ncon, nnpg;
  long long nz;
};

// DJACAB (djac.f:1-139) + DABMKISOB25 (dstiff25.f:1-203) of element e for
// inversion anchor p, into shared memory as COMPLEX*8
// CARG = CMPLX(DCMPLX(DMD,0) + DKD) [75][75]: carg0 holds the first variable
// (alpha when lisp), carg1 beta when both.  sm: SHG tables and per-point
// coefficients.  Every thread of the CTA calls it; it ends with a barrier.
__device__ __forceinline__ void dabm_carg(const MeshView &mv, const DevTables &dt, int e, int p,
                                          double wpy, double wpy2, int lisp, int liss, double *sm,
                                          float2 *carg0, float2 *carg1, int *err) {
  double *shx = sm, *shz = sm + kNq * kNen, *shn = sm + 2 * kNq * kNen;
  double *qc = sm + 3 * kNq * kNen;  // [kNq][8]
  const int t = threadIdx.x;
  const int4 ie = mv.ieng[e];
  if (t < kNq) {
    const int q = t, intx = q % kNint, intz = q / kNint;
    QGeo g;
    if (!quad_geo(mv, dt, ie, q, false, g)) atomicCAS(err, 0, e + 1);
    // DJACAB (djac.f:90-110)
    const int il[4] = {ie.x - 1, ie.y - 1, ie.z - 1, ie.w - 1};
    double dab1 = 0.0, dab2 = 0.0;
    for (int ia = 0; ia < 4; ia++) {
      double alpha = 0.0, beta = 0.0;
      if (il[ia] == p) {
        alpha = sqrt((mv.lam[p] + 2.0 * mv.mu[p]) / mv.rho[p]);
        beta = sqrt(mv.mu[p] / mv.rho[p]);
      }
      dab1 = dab1 + 2.0 * alpha * dt.sf[4 * q + ia];
      dab2 = dab2 + 2.0 * beta * dt.sf[4 * q + ia];
    }
    double *c = qc + 8 * q;
    c[0] = g.dxdxi; c[1] = g.dxdeta; c[2] = g.dzdxi; c[3] = g.dzdeta; c[4] = g.rjac;
    double weight = dt.wts[intx] * dt.wts[intz] * g.rjac;
    c[5] = dab1 * weight;  // DALPHA
    c[6] = dab2 * weight;  // DBETA
  }
  __syncthreads();
  for (int idx = t; idx < kNq * kNen; idx += kRefThreads) {
    const int q = idx / kNen;
    const double *c = qc + 8 * q;
    const double *sl = dt.shl + 3 * (size_t)idx;
    double drnxi = sl[0], drneta = sl[1];
    shx[idx] = (drnxi * c[3] - drneta * c[2]) / c[4];
    shz[idx] = -(drnxi * c[1] - drneta * c[0]) / c[4];
    shn[idx] = sl[2];
  }
  __syncthreads();
  if (t < kNab) {
    const int a = t / kNen, b = t % kNen;
    // alpha: DMDA(1,1); DKDA real 00 02 20 22, imaginary 01 10 12 21
    double ma11 = 0.0, ra00 = 0.0, ra02 = 0.0, ra20 = 0.0, ra22 = 0.0;
    double ia01 = 0.0, ia10 = 0.0, ia12 = 0.0, ia21 = 0.0;
    // beta: DMDB(0,0) (= DMDB(2,2)); DKDB real 00 02 11 20 22, imaginary 01 10 12 21
    double mb00 = 0.0, rb00 = 0.0, rb02 = 0.0, rb11 = 0.0, rb20 = 0.0, rb22 = 0.0;
    double ib01 = 0.0, ib10 = 0.0, ib12 = 0.0, ib21 = 0.0;
    for (int intx = 0; intx < kNint; intx++)
      for (int intz = 0; intz < kNint; intz++) {
        const int q = intx + kNint * intz;
        const double dalpha = qc[8 * q + 5], dbeta = qc[8 * q + 6];
        const double phib = shn[q * kNen + b], phibx = shx[q * kNen + b], phibz = shz[q * kNen + b];
        const double phia = shn[q * kNen + a], phiax = shx[q * kNen + a], phiaz = shz[q * kNen + a];
        if (lisp) {
          const double dmassda = wpy2 * dalpha;
          const double dmdat1 = dmassda * phib;
          const double dk11da = dalpha * phibx, dk13da = dalpha * phibz;
          const double dk31da = dalpha * phibx, dk33da = dalpha * phibz;
          const double dk12da = wpy * dalpha * phib, dk21da = wpy * dalpha * phibx;
          const double dk23da = wpy * dalpha * phibz, dk32da = wpy * dalpha * phib;
          ma11 = ma11 + dmdat1 * phia;
          ra00 = ra00 + phiax * dk11da;
          ia01 = ia01 - phiax * dk12da;
          ra02 = ra02 + phiax * dk13da;
          ia10 = ia10 + phia * dk21da;
          ia12 = ia12 + phia * dk23da;
          ra20 = ra20 + phiaz * dk31da;
          ia21 = ia21 - phiaz * dk32da;
          ra22 = ra22 + phiaz * dk33da;
        }
        if (liss) {
          const double dmassdb = wpy2 * dbeta;
          const double dmdbt1 = dmassdb * phib;
          const double dk11dbt1 = dbeta * phibz;
          const double dk13dbt1 = dbeta * phibx, dk13dbt2 = -(2.0 * dbeta * phibz);
          const double dk22dbt1 = dbeta * phibx, dk22dbt2 = dbeta * phibz;
          const double dk31dbt1 = dbeta * phibz, dk31dbt2 = -(2.0 * dbeta * phibx);
          const double dk33dbt1 = dbeta * phibx;
          const double dk12dbt1 = 2.0 * wpy * dbeta * phib, dk12dbt2 = wpy * dbeta * phibx;
          const double dk21dbt1 = 2.0 * wpy * dbeta * phibx, dk21dbt2 = wpy * dbeta * phib;
          const double dk23dbt1 = 2.0 * wpy * dbeta * phibz, dk23dbt2 = wpy * dbeta * phib;
          const double dk32dbt1 = 2.0 * wpy * dbeta * phib, dk32dbt2 = wpy * dbeta * phibz;
          mb00 = mb00 + dmdbt1 * phia;
          rb00 = rb00 + phiaz * dk11dbt1;
          ib01 = ib01 + (phiax * dk12dbt1 + phia * dk12dbt2);
          rb02 = rb02 + (phiaz * dk13dbt1 + phiax * dk13dbt2);
          ib10 = ib10 - (phia * dk21dbt1 + phiax * dk21dbt2);
          rb11 = rb11 + (phiax * dk22dbt1 + phiaz * dk22dbt2);
          ib12 = ib12 - (phia * dk23dbt1 + phiaz * dk23dbt2);
          rb20 = rb20 + (phiax * dk31dbt1 + phiaz * dk31dbt2);
          ib21 = ib21 + (phiaz * dk32dbt1 + phia * dk32dbt2);
          rb22 = rb22 + phiax * dk33dbt1;
        }
      }
    const int ipe = 3 * a, iqe = 3 * b;
    auto put = [&](float2 *cg, int i, int j, double re, double im) {
      cg[(size_t)(ipe + i) * kNee + iqe + j] =
          make_float2(__double2float_rn(re), __double2float_rn(0.0 + im));
    };
    float2 *cb = carg0;
    if (lisp) {
      put(cb, 0, 0, 0.0 + ra00, 0.0);
      put(cb, 0, 1, 0.0 + 0.0, ia01);
      put(cb, 0, 2, 0.0 + ra02, 0.0);
      put(cb, 1, 0, 0.0 + 0.0, ia10);
      put(cb, 1, 1, ma11 + 0.0, 0.0);
      put(cb, 1, 2, 0.0 + 0.0, ia12);
      put(cb, 2, 0, 0.0 + ra20, 0.0);
      put(cb, 2, 1, 0.0 + 0.0, ia21);
      put(cb, 2, 2, 0.0 + ra22, 0.0);
      cb = carg1;
    }
    if (liss) {
      put(cb, 0, 0, mb00 + rb00, 0.0);
      put(cb, 0, 1, 0.0 + 0.0, ib01);
      put(cb, 0, 2, 0.0 + rb02, 0.0);
      put(cb, 1, 0, 0.0 + 0.0, ib10);
      put(cb, 1, 1, 0.0 + rb11, 0.0);
      put(cb, 1, 2, 0.0 + 0.0, ib12);
      put(cb, 2, 0, 0.0 + rb20, 0.0);
      put(cb, 2, 1, 0.0 + 0.0, ib21);
      put(cb, 2, 2, mb00 + rb22, 0.0);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kRefThreads, 1)
    k_ref_vforce2(MeshView mv, DevTables dt, VfArgs va, const int *__restrict__ lm,
                  const int *__restrict__ anchor_of_col, const int *__restrict__ mconn,
                  const int *__restrict__ jcsc, const int *__restrict__ icsc,
                  const float2 *__restrict__ wave, float2 *__restrict__ fmat,
                  int *__restrict__ err) {
  extern __shared__ double sm[];
  float2 *carg0 = reinterpret_cast<float2 *>(sm + 3 * kNq * kNen + 8 * kNq);  // [75][75] first variable
  float2 *carg1 = carg0 + kNee * kNee;  // [75][75] beta when 'PS'
  const int col = blockIdx.x, t = threadIdx.x;
  const int p = anchor_of_col[col];
  const int i1 = jcsc[col] - 1, i2 = jcsc[col + 1] - 1, nnzrow = i2 - i1;
  const int nvar = va.lisp + va.liss;
  for (int v = 0; v < nvar; v++)
    for (int k = t; k < nnzrow; k += kRefThreads) fmat[v * va.nz + i1 + k] = make_float2(0.0f, 0.0f);
  const double wpy = va.omega * va.py, wpy2 = ipow2(va.omega * va.py);
  __syncthreads();
  for (int ic = 0; ic < va.ncon; ic++) {
    const int e1 = mconn[p + (size_t)va.nnpg * ic];
    if (e1 <= 0) break;
    const int e = e1 - 1;
    dabm_carg(mv, dt, e, p, wpy, wpy2, va.lisp, va.liss, sm, carg0, carg1, err);
    if (t < kNee) {
      const int ipe = t;
      const int *lme = lm + (size_t)e * kNee;
      const int idof = lme[ipe];
      if (idof > 0) {
        int lo = 0, hi = nnzrow - 1, inz = -1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1, v = icsc[i1 + mid];
          if (v == idof) { inz = mid; break; }
          if (v < idof) lo = mid + 1;
          else hi = mid - 1;
        }
        if (inz < 0) {
          atomicCAS(err, 0, -(col + 1));
        } else {
          for (int v = 0; v < nvar; v++) {
            const float2 *cg = v == 0 ? carg0 : carg1;
            float2 *f = fmat + v * va.nz + i1 + inz;
            float fr = f->x, fi = f->y;
            for (int iqe = 0; iqe < kNee; iqe++) {
              const int jdof = lme[iqe];
              if (jdof <= 0) continue;
              const float2 cv = cg[(size_t)ipe * kNee + iqe], wv = wave[jdof - 1];
              cfl t1 = cmulf(cfl{cv.x, cv.y}, cfl{wv.x, wv.y});
              fr = fr + t1.re;
              fi = fi + t1.im;
            }
            *f = make_float2(fr, fi);
          }
        }
      }
    }
    __syncthreads();
  }
}

// MET225_MOD (qpmfree.f90:1000-1250): one CTA per CSC column (inversion
// anchor).  For each connected element (MCONN order) the DABMKISOB25 blocks
// are integrated as in VFORCE25_2; 75 threads then add, row by row,
// (CWGHT * CARG) * WAVE and (CWGHT * CARG) * ALPHA into the shared-memory
// columns T1, T2 of each variable (nulled inside the element loop, as the
// reference does, unless accumulate).  Finally one thread per (variable,
// buffer) forms PBUF1 -= REAL(CONJG(T1) * NU), PBUF2 -= REAL(CONJG(T2) *
// ADJLAM) over the column's rows in order.  p1buf, p2buf: [ncol * nvar],
// entry col * nvar + v (alpha before beta).
struct MetArgs {
  double omega, py;
  int lisp, liss, ncon, nnpg, maxrow, accumulate;
};

__global__ void __launch_bounds__(kRefThreads, 1)
    k_ref_met225(MeshView mv, DevTables dt, MetArgs ma, const int *__restrict__ lm,
                 const int *__restrict__ anchor_of_col, const int *__restrict__ mconn,
                 const double *__restrict__ elem_wts, const int *__restrict__ jcsc,
                 const int *__restrict__ icsc, const float2 *__restrict__ adjlam,
                 const float2 *__restrict__ nu, const float2 *__restrict__ alpha,
                 const float2 *__restrict__ wave, float *__restrict__ p1buf,
                 float *__restrict__ p2buf, int *__restrict__ err) {
  extern __shared__ double sm[];
  float2 *carg0 = reinterpret_cast<float2 *>(sm + 3 * kNq * kNen + 8 * kNq);
  float2 *carg1 = carg0 + kNee * kNee;
  float2 *t1 = carg1 + kNee * kNee;  // [2][maxrow]
  float2 *t2 = t1 + 2 * ma.maxrow;   // [2][maxrow]
  const int col = blockIdx.x, t = threadIdx.x;
  const int p = anchor_of_col[col];
  const int i1 = jcsc[col] - 1, i2 = jcsc[col + 1] - 1, nnzrow = i2 - i1;
  const int nvar = ma.lisp + ma.liss;
  const double wpy = ma.omega * ma.py, wpy2 = ipow2(ma.omega * ma.py);
  for (int k = t; k < 2 * ma.maxrow; k += kRefThreads) {
    t1[k] = make_float2(0.0f, 0.0f);
    t2[k] = make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  for (int ic = 0; ic < ma.ncon; ic++) {
    const int e1 = mconn[p + (size_t)ma.nnpg * ic];
    if (e1 <= 0) break;
    const int e = e1 - 1;
    dabm_carg(mv, dt, e, p, wpy, wpy2, ma.lisp, ma.liss, sm, carg0, carg1, err);
    if (!ma.accumulate) {
      for (int k = t; k < 2 * ma.maxrow; k += kRefThreads) {
        t1[k] = make_float2(0.0f, 0.0f);
        t2[k] = make_float2(0.0f, 0.0f);
      }
      __syncthreads();
    }
    if (t < kNee) {
      const int ipe = t;
      const int *lme = lm + (size_t)e * kNee;
      const int idof = lme[ipe];
      if (idof > 0) {
        int lo = 0, hi = nnzrow - 1, inz = -1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1, v = icsc[i1 + mid];
          if (v == idof) { inz = mid; break; }
          if (v < idof) lo = mid + 1;
          else hi = mid - 1;
        }
        if (inz < 0) {
          atomicCAS(err, 0, -(col + 1));
        } else {
          const cfl cwght{__double2float_rn(elem_wts[e]), 0.0f};
          for (int v = 0; v < nvar; v++) {
            const float2 *cg = v == 0 ? carg0 : carg1;
            float2 *r1 = t1 + v * ma.maxrow + inz, *r2 = t2 + v * ma.maxrow + inz;
            float ar = r1->x, ai = r1->y, br = r2->x, bi = r2->y;
            for (int iqe = 0; iqe < kNee; iqe++) {
              const int jdof = lme[iqe];
              if (jdof <= 0) continue;
              const float2 cv = cg[(size_t)ipe * kNee + iqe];
              const cfl cw = cmulf(cwght, cfl{cv.x, cv.y});
              const float2 wv = wave[jdof - 1], av = alpha[jdof - 1];
              const cfl a1 = cmulf(cw, cfl{wv.x, wv.y}), a2 = cmulf(cw, cfl{av.x, av.y});
              ar = ar + a1.re;
              ai = ai + a1.im;
              br = br + a2.re;
              bi = bi + a2.im;
            }
            *r1 = make_float2(ar, ai);
            *r2 = make_float2(br, bi);
          }
        }
      }
    }
    __syncthreads();
  }
  if (t < 2 * nvar) {
    const int v = t >> 1, which = t & 1;
    const float2 *tv = (which ? t2 : t1) + v * ma.maxrow;
    const float2 *x = which ? adjlam : nu;
    float acc = 0.0f;
    for (int k = 0; k < nnzrow; k++) {
      const float2 a = tv[k], b = x[icsc[i1 + k] - 1];
      const float ar = a.x, ai = -a.y;  // CONJG
      acc = acc - (ar * b.x - ai * b.y);
    }
    (which ? p2buf : p1buf)[(size_t)col * nvar + v] = acc;
  }
}

// CADJ_NU_ALPHA (qpmfree.f90:622-996) without its solves, in three passes so
// that every FP32 sum runs in the reference's order:
//  1. one CTA per (anchor column, connected element) pair: the DABMKISOB25
//     blocks (the first-derivative blocks of DABM2KISOB25 are the same
//     arithmetic) times CWGHT = CMPLX(SNGL(ELEM_WTS) * V(ia35), 0), stored as
//     W[pair][v][75][75];
//  2. one thread per DOF d walks d's (pair, local index l) list in pair order:
//     RHSALP(d) += W_v(l, iqe) * WAVE(JDOF) over iqe, v, and
//     RHSBNU(d) += ADJLAM(IDOF) * CONJG(W_v(ipe, l)) over ipe, v;
//  3. one CTA per column: TEMP_v(row) += W_v(ipe, iqe) * WAVE(JDOF) over the
//     column's elements (nulled per element unless accumulate), then
//     P3(ia35) -= REAL(CONJG(TEMP_v) * ADJLAM) over the column's rows.
struct CadjArgs {
  double omega, py;
  int lisp, liss, nnpg, maxrow, accumulate, ndof;
};

__global__ void __launch_bounds__(kRefThreads, 1)
    k_ref_cadj_w(MeshView mv, DevTables dt, CadjArgs ca, const int *__restrict__ anchor_of_col,
                 const int *__restrict__ pair_col, const int *__restrict__ pair_elem,
                 const double *__restrict__ elem_wts, const float *__restrict__ v,
                 float2 *__restrict__ wout, int *__restrict__ err) {
  extern __shared__ double sm[];
  float2 *carg0 = reinterpret_cast<float2 *>(sm + 3 * kNq * kNen + 8 * kNq);
  float2 *carg1 = carg0 + kNee * kNee;
  const int k = blockIdx.x, col = pair_col[k], e = pair_elem[k];
  const int p = anchor_of_col[col];
  const int nvar = ca.lisp + ca.liss;
  const double wpy = ca.omega * ca.py, wpy2 = ipow2(ca.omega * ca.py);
  dabm_carg(mv, dt, e, p, wpy, wpy2, ca.lisp, ca.liss, sm, carg0, carg1, err);
  const float swt = __double2float_rn(elem_wts[e]);
  for (int var = 0; var < nvar; var++) {
    const cfl cwght{swt * v[(size_t)col * nvar + var], 0.0f};
    const float2 *cg = var == 0 ? carg0 : carg1;
    float2 *wo = wout + ((size_t)k * nvar + var) * kNee * kNee;
    for (int i = threadIdx.x; i < kNee * kNee; i += kRefThreads) {
      const cfl w = cmulf(cwght, cfl{cg[i].x, cg[i].y});
      wo[i] = make_float2(w.re, w.im);
    }
  }
}

__global__ void k_ref_cadj_rhs(CadjArgs ca, const int *__restrict__ lm,
                               const int *__restrict__ pair_elem, const int *__restrict__ dptr,
                               const int *__restrict__ dent, const float2 *__restrict__ w,
                               const float2 *__restrict__ adjlam, const float2 *__restrict__ wave,
                               float2 *__restrict__ rhsbnu, float2 *__restrict__ rhsalp) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= ca.ndof) return;
  const int nvar = ca.lisp + ca.liss;
  float br = 0.0f, bi = 0.0f, ar = 0.0f, ai = 0.0f;
  for (int j = dptr[d]; j < dptr[d + 1]; j++) {
    const int k = dent[j] >> 7, l = dent[j] & 127;
    const int *lme = lm + (size_t)pair_elem[k] * kNee;
    const float2 *wk = w + (size_t)k * nvar * kNee * kNee;
    // RHSALP(d): row l of each variable's block
    for (int iqe = 0; iqe < kNee; iqe++) {
      const int jdof = lme[iqe];
      if (jdof <= 0) continue;
      const float2 x = wave[jdof - 1];
      for (int var = 0; var < nvar; var++) {
        const float2 c = wk[(size_t)var * kNee * kNee + l * kNee + iqe];
        const cfl t = cmulf(cfl{c.x, c.y}, cfl{x.x, x.y});
        ar = ar + t.re;
        ai = ai + t.im;
      }
    }
    // RHSBNU(d): column l of each variable's block
    for (int ipe = 0; ipe < kNee; ipe++) {
      const int idof = lme[ipe];
      if (idof <= 0) continue;
      const float2 x = adjlam[idof - 1];
      for (int var = 0; var < nvar; var++) {
        const float2 c = wk[(size_t)var * kNee * kNee + ipe * kNee + l];
        const cfl t = cmulf(cfl{x.x, x.y}, cfl{c.x, -c.y});
        br = br + t.re;
        bi = bi + t.im;
      }
    }
  }
  rhsalp[d] = make_float2(ar, ai);
  rhsbnu[d] = make_float2(br, bi);
}

__global__ void __launch_bounds__(128)
    k_ref_cadj_p3(CadjArgs ca, const int *__restrict__ lm, const int *__restrict__ col_pair0,
                  const int *__restrict__ pair_elem, const int *__restrict__ jcsc,
                  const int *__restrict__ icsc, const float2 *__restrict__ w,
                  const float2 *__restrict__ adjlam, const float2 *__restrict__ wave,
                  float *__restrict__ p3, int *__restrict__ err) {
  extern __shared__ float2 temp[];  // [2][maxrow]
  const int col = blockIdx.x, t = threadIdx.x;
  const int i1 = jcsc[col] - 1, i2 = jcsc[col + 1] - 1, nnzrow = i2 - i1;
  const int nvar = ca.lisp + ca.liss;
  for (int k = t; k < 2 * ca.maxrow; k += blockDim.x) temp[k] = make_float2(0.0f, 0.0f);
  __syncthreads();
  for (int k = col_pair0[col]; k < col_pair0[col + 1]; k++) {
    if (!ca.accumulate) {
      for (int i = t; i < 2 * ca.maxrow; i += blockDim.x) temp[i] = make_float2(0.0f, 0.0f);
      __syncthreads();
    }
    const int *lme = lm + (size_t)pair_elem[k] * kNee;
    if (t < kNee) {
      const int idof = lme[t];
      if (idof > 0) {
        int lo = 0, hi = nnzrow - 1, inz = -1;
        while (lo <= hi) {
          int mid = (lo + hi) >> 1, v = icsc[i1 + mid];
          if (v == idof) { inz = mid; break; }
          if (v < idof) lo = mid + 1;
          else hi = mid - 1;
        }
        if (inz < 0) {
          atomicCAS(err, 0, -(col + 1));
        } else {
          for (int var = 0; var < nvar; var++) {
            const float2 *wr = w + ((size_t)k * nvar + var) * kNee * kNee + (size_t)t * kNee;
            float2 *r = temp + var * ca.maxrow + inz;
            float xr = r->x, xi = r->y;
            for (int iqe = 0; iqe < kNee; iqe++) {
              const int jdof = lme[iqe];
              if (jdof <= 0) continue;
              const float2 c = wr[iqe], x = wave[jdof - 1];
              const cfl s = cmulf(cfl{c.x, c.y}, cfl{x.x, x.y});
              xr = xr + s.re;
              xi = xi + s.im;
            }
            *r = make_float2(xr, xi);
          }
        }
      }
    }
    __syncthreads();
  }
  if (t < nvar) {
    const float2 *tv = temp + t * ca.maxrow;
    float acc = 0.0f;
    for (int k = 0; k < nnzrow; k++) {
      const float2 a = tv[k], b = adjlam[icsc[i1 + k] - 1];
      const float xr = a.x, xi = -a.y;  // CONJG
      acc = acc - (xr * b.x - xi * b.y);
    }
    p3[(size_t)col * nvar + t] = acc;
  }
}

// PCHADJ (pchadj.f90:1-330) after the Green's-function solve: one CTA per
// inversion anchor column.  Threads over (irhs, v) form
// JACL(irhs, v) = sum_rows G((irhs-1)*NDOF + JDOF) * FMAT(row, v) in row order
// (pchadj.f90:241-246) into shared memory (and jacl when given); then one
// thread per (iv, jv) forms REAL(sum_l CONJG(JACL(l, iv)) * JACL(l, jv)) in
// the reference BLAS order (CGEMM 'C','N', ALPHA = 1) and adds it to HESSB
// (pchadj.f90:274-300, 312-323).
__global__ void __launch_bounds__(256)
    k_ref_pchadj(int nvinv, long long nz, int ndof, int nrhs, const int *__restrict__ jcsc,
                 const int *__restrict__ icsc, const float2 *__restrict__ grns,
                 const float2 *__restrict__ fmat, float *__restrict__ hessb,
                 float2 *__restrict__ jacl) {
  extern __shared__ float2 jl[];  // [nrhs][nvinv]
  const int col = blockIdx.x;
  const int i1 = jcsc[col] - 1, i2 = jcsc[col + 1] - 1;
  for (int idx = threadIdx.x; idx < nrhs * nvinv; idx += blockDim.x) {
    const int irhs = idx / nvinv, v = idx % nvinv;
    const float2 *gr = grns + (size_t)irhs * ndof;
    const float2 *fv = fmat + (size_t)v * nz;
    float ar = 0.0f, ai = 0.0f;
    for (int i = i1; i < i2; i++) {
      const int jdof = icsc[i];
      if (jdof == 0) continue;
      const float2 g = gr[jdof - 1], f = fv[i];
      const cfl t = cmulf(cfl{g.x, g.y}, cfl{f.x, f.y});
      ar = ar + t.re;
      ai = ai + t.im;
    }
    jl[idx] = make_float2(ar, ai);
    if (jacl) jacl[((size_t)col * nvinv + v) * nrhs + irhs] = make_float2(ar, ai);
  }
  __syncthreads();
  if (threadIdx.x < nvinv * nvinv) {
    const int iv = threadIdx.x / nvinv, jv = threadIdx.x % nvinv;
    float tr = 0.0f, ti = 0.0f;
    for (int l = 0; l < nrhs; l++) {
      const float2 a = jl[l * nvinv + iv], b = jl[l * nvinv + jv];
      const cfl t = cmulf(cfl{a.x, -a.y}, cfl{b.x, b.y});
      tr = tr + t.re;
      ti = ti + t.im;
    }
    const cfl h = cmulf(cfl{1.0f, 0.0f}, cfl{tr, ti});
    const float hb = 0.0f + h.re;
    float *y = hessb + ((size_t)col * nvinv + iv) * nvinv + jv;
    *y = *y + 1.0f * hb;
  }
}

// ADJFLAM_DIST (adjgrad.f90:128-139) + SAXPY(-1) into GRADL (adjgrad.f90:76)
__global__ void k_ref_adjflam(int ncol, const int *__restrict__ jcsc, const int *__restrict__ icsc,
                              const float2 *__restrict__ fmat, const float2 *__restrict__ lam,
                              float *__restrict__ gradl) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncol) return;
  float v = 0.0f;
  for (int i = jcsc[k] - 1; i < jcsc[k + 1] - 1; i++) {
    const float2 f = fmat[i], l = lam[icsc[i] - 1];
    const float fr = f.x, fi = -f.y;
    v = v - (fr * l.x - fi * l.y);
  }
  gradl[k] = gradl[k] + (-1.0f) * v;
}

static size_t ref_smem() {
  return sizeof(double) * (3 * kNq * kNen + 8 * kNq) + sizeof(float2) * kNee * kNee;
}

cudaError_t launch_ref_cfmat(Ctx *c, int lisp, double vpvs, double omega, double py,
                             const float *wave, int accumulate, cudaStream_t st) {
  RefArgs ra;
  ra.omega = omega;
  ra.py = py;
  ra.vpvs2 = vpvs * vpvs;
  ra.lisp = lisp;
  ra.accumulate = accumulate;
  ra.ncon = c->rg.ncon;
  ra.nnpg = c->nnpg;
  cudaError_t e = cudaFuncSetAttribute(k_ref_cfmat, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ref_smem());
  if (e) return e;
  k_ref_cfmat<<<c->rg.nnpinv, kRefThreads, ref_smem(), st>>>(
      c->mv, c->dt, ra, c->d_lm, c->d_rg_anchor, c->d_mconn, c->d_elem_wts, c->d_jcsc, c->d_icsc,
      (const float2 *)wave, c->d_fmat, c->d_err);
  return cudaGetLastError();
}

static size_t vforce2_smem() {
  return sizeof(double) * (3 * kNq * kNen + 8 * kNq) + sizeof(float2) * 2 * kNee * kNee;
}

cudaError_t launch_ref_vforce2(Ctx *c, int lisp, int liss, double omega, double py,
                               const float *wave, float *fmat, cudaStream_t st) {
  VfArgs va;
  va.omega = omega;
  va.py = py;
  va.lisp = lisp;
  va.liss = liss;
  va.ncon = c->rg.ncon;
  va.nnpg = c->nnpg;
  va.nz = c->rg.nz;
  cudaError_t e = cudaFuncSetAttribute(k_ref_vforce2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)vforce2_smem());
  if (e) return e;
  k_ref_vforce2<<<c->rg.nnpinv, kRefThreads, vforce2_smem(), st>>>(
      c->mv, c->dt, va, c->d_lm, c->d_rg_anchor, c->d_mconn, c->d_jcsc, c->d_icsc,
      (const float2 *)wave, (float2 *)fmat, c->d_err);
  return cudaGetLastError();
}

cudaError_t launch_ref_met225(Ctx *c, int lisp, int liss, double omega, double py,
                              const float *adjlam, const float *nu, const float *alpha,
                              const float *wave, int accumulate, float *p1buf, float *p2buf,
                              cudaStream_t st) {
  MetArgs ma;
  ma.omega = omega;
  ma.py = py;
  ma.lisp = lisp;
  ma.liss = liss;
  ma.ncon = c->rg.ncon;
  ma.nnpg = c->nnpg;
  ma.accumulate = accumulate;
  ma.maxrow = 1;
  for (int k = 0; k < c->rg.nnpinv; k++)
    ma.maxrow = std::max(ma.maxrow, c->rg.jcsc[k + 1] - c->rg.jcsc[k]);
  const size_t smem = vforce2_smem() + sizeof(float2) * 4 * (size_t)ma.maxrow;
  cudaError_t e = cudaFuncSetAttribute(k_ref_met225, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  k_ref_met225<<<c->rg.nnpinv, kRefThreads, smem, st>>>(
      c->mv, c->dt, ma, c->d_lm, c->d_rg_anchor, c->d_mconn, c->d_elem_wts, c->d_jcsc, c->d_icsc,
      (const float2 *)adjlam, (const float2 *)nu, (const float2 *)alpha, (const float2 *)wave,
      p1buf, p2buf, c->d_err);
  return cudaGetLastError();
}

// Pair list and per-DOF contribution lists of CADJ_NU_ALPHA (host, once).
int prepare_cadj(Ctx *c, std::string *msg) {
  if (c->cadj_npairs >= 0) return 0;
  const RefGradSetup &rg = c->rg;
  std::vector<int> pcol, pelem, col0(rg.nnpinv + 1, 0);
  for (int col = 0; col < rg.nnpinv; col++) {
    col0[col] = (int)pcol.size();
    const int p = rg.anchor_of_col[col];
    for (int ic = 0; ic < rg.ncon; ic++) {
      const int e1 = rg.mconn[p + (size_t)c->nnpg * ic];
      if (e1 <= 0) break;
      pcol.push_back(col);
      pelem.push_back(e1 - 1);
    }
  }
  const int np = (int)pcol.size();
  col0[rg.nnpinv] = np;
  if ((long long)np >= (1LL << 24)) {
    *msg = "cadj_nu_alpha: more than 2^24 (anchor, element) pairs";
    return FEM25_ERR_UNSUPPORTED;
  }
  std::vector<int> cnt(c->ndof + 1, 0);
  for (int k = 0; k < np; k++)
    for (int l = 0; l < kNee; l++) {
      const int d = c->h_lm[(size_t)pelem[k] * kNee + l];
      if (d > 0) cnt[d - 1 + 1]++;
    }
  for (int d = 0; d < c->ndof; d++) cnt[d + 1] += cnt[d];
  std::vector<int> ent(cnt[c->ndof]), cur(cnt.begin(), cnt.end() - 1);
  for (int k = 0; k < np; k++)
    for (int l = 0; l < kNee; l++) {
      const int d = c->h_lm[(size_t)pelem[k] * kNee + l];
      if (d > 0) ent[cur[d - 1]++] = (k << 7) | l;
    }
  cudaError_t e = cudaSuccess;
  auto up = [&](int **dst, const std::vector<int> &src) {
    if ((e = cudaMalloc(dst, sizeof(int) * std::max<size_t>(1, src.size())))) return false;
    if (!src.empty() &&
        (e = cudaMemcpy(*dst, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice)))
      return false;
    return true;
  };
  if (!up(&c->d_cadj_col0, col0) || !up(&c->d_cadj_pair_col, pcol) ||
      !up(&c->d_cadj_pair_elem, pelem) || !up(&c->d_cadj_dptr, cnt) ||
      !up(&c->d_cadj_dent, ent)) {
    *msg = std::string("cadj_nu_alpha: ") + cudaGetErrorString(e);
    return FEM25_ERR_ALLOC;
  }
  c->cadj_npairs = np;
  return 0;
}

cudaError_t launch_ref_cadj(Ctx *c, int lisp, int liss, double omega, double py, const float *v,
                            const float *adjlam, const float *wave, int accumulate, float *rhsbnu,
                            float *rhsalp, float *p3, cudaStream_t st) {
  CadjArgs ca;
  ca.omega = omega;
  ca.py = py;
  ca.lisp = lisp;
  ca.liss = liss;
  ca.nnpg = c->nnpg;
  ca.accumulate = accumulate;
  ca.ndof = c->ndof;
  ca.maxrow = 1;
  for (int k = 0; k < c->rg.nnpinv; k++)
    ca.maxrow = std::max(ca.maxrow, c->rg.jcsc[k + 1] - c->rg.jcsc[k]);
  const int nvar = lisp + liss;
  const size_t wbytes = sizeof(float2) * (size_t)std::max(1, c->cadj_npairs) * nvar * kNee * kNee;
  cudaError_t e;
  if (wbytes > c->cadj_w_cap) {
    if ((e = cudaStreamSynchronize(st))) return e;
    if (c->d_cadj_w) cudaFree(c->d_cadj_w);
    c->d_cadj_w = nullptr;
    c->cadj_w_cap = 0;
    if ((e = cudaMalloc(&c->d_cadj_w, wbytes))) return e;
    c->cadj_w_cap = wbytes;
  }
  if ((e = cudaFuncSetAttribute(k_ref_cadj_w, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)vforce2_smem())))
    return e;
  if (c->cadj_npairs > 0)
    k_ref_cadj_w<<<c->cadj_npairs, kRefThreads, vforce2_smem(), st>>>(
        c->mv, c->dt, ca, c->d_rg_anchor, c->d_cadj_pair_col, c->d_cadj_pair_elem, c->d_elem_wts,
        v, c->d_cadj_w, c->d_err);
  k_ref_cadj_rhs<<<(c->ndof + 127) / 128, 128, 0, st>>>(
      ca, c->d_lm, c->d_cadj_pair_elem, c->d_cadj_dptr, c->d_cadj_dent, c->d_cadj_w,
      (const float2 *)adjlam, (const float2 *)wave, (float2 *)rhsbnu, (float2 *)rhsalp);
  k_ref_cadj_p3<<<c->rg.nnpinv, 128, sizeof(float2) * 2 * ca.maxrow, st>>>(
      ca, c->d_lm, c->d_cadj_col0, c->d_cadj_pair_elem, c->d_jcsc, c->d_icsc, c->d_cadj_w,
      (const float2 *)adjlam, (const float2 *)wave, p3, c->d_err);
  return cudaGetLastError();
}

cudaError_t launch_ref_pchadj(Ctx *c, int nvinv, int nrhs, const float *grns, const float *fmat,
                              float *hessb, float *jacl, cudaStream_t st) {
  const size_t smem = sizeof(float2) * (size_t)nrhs * nvinv;
  cudaError_t e = cudaFuncSetAttribute(k_ref_pchadj, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  k_ref_pchadj<<<c->rg.nnpinv, 256, smem, st>>>(nvinv, c->rg.nz, c->ndof, nrhs, c->d_jcsc,
                                                c->d_icsc, (const float2 *)grns,
                                                (const float2 *)fmat, hessb, (float2 *)jacl);
  return cudaGetLastError();
}

cudaError_t launch_ref_adjflam(Ctx *c, const float *adjlam, float *gradl, cudaStream_t st) {
  int n = c->rg.nnpinv;
  k_ref_adjflam<<<(n + 255) / 256, 256, 0, st>>>(n, c->d_jcsc, c->d_icsc, c->d_fmat,
                                                 (const float2 *)adjlam, gradl);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// gradient post-processing of FUNCGRADH25 (funcgradh.f90:436-443)
// ---------------------------------------------------------------------------
// WTGRAD (gengmask.f90:384-416): GRAD(IA35) = GRAD(IA35) * WGRAD(IA35)
__global__ void k_wtgrad(int na35, const float *__restrict__ wgrad, float *__restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < na35) grad[i] = grad[i] * wgrad[i];
}

cudaError_t launch_wtgrad(int na35, const float *wgrad, float *grad, cudaStream_t st) {
  k_wtgrad<<<(na35 + 255) / 256, 256, 0, st>>>(na35, wgrad, grad);
  return cudaGetLastError();
}

// One cascade of AVGRAD / AVGRAD8 (gengmask.f90:1202-1332), one thread per
// anchor INPG: the mean of the gradient over the inversion anchors of every
// element connected to INPG (MCONN order, anchors IA = 1..4 of each
// element, counted with repetition as in the reference), written to `out`;
// anchors outside the inversion and entries without neighbours keep `in`.
template <typename T>
__global__ void k_avgrad(int nnpg, int ncon, int nvinv, const int *__restrict__ maskg,
                         const int *__restrict__ mconn, const int4 *__restrict__ ieng,
                         const T *__restrict__ in, T *__restrict__ out) {
  const int inpg = blockIdx.x * blockDim.x + threadIdx.x;
  if (inpg >= nnpg) return;
  const int inpinv = maskg[inpg];
  if (inpinv <= 0) return;
  T xavg[2] = {T(0), T(0)};
  int navg[2] = {0, 0};
  for (int icon = 0; icon < ncon; icon++) {
    const int ielem = mconn[inpg + (size_t)nnpg * icon];
    if (ielem == 0) break;
    const int4 ie = ieng[ielem - 1];
    const int an[4] = {ie.x, ie.y, ie.z, ie.w};
    for (int ia = 0; ia < 4; ia++) {
      const int jnpg = an[ia];
      if (jnpg == 0) break;
      const int jnpinv = maskg[jnpg - 1];
      if (jnpinv > 0)
        for (int iv = 0; iv < nvinv; iv++) {
          xavg[iv] = xavg[iv] + in[(size_t)(jnpinv - 1) * nvinv + iv];
          navg[iv] = navg[iv] + 1;
        }
    }
  }
  for (int iv = 0; iv < nvinv; iv++) {
    const size_t ia35 = (size_t)(inpinv - 1) * nvinv + iv;
    if (navg[iv] > 0) out[ia35] = xavg[iv] / (T)navg[iv];
  }
}

// NCASC cascades; each starts from a copy of the gradient (SCOPY / DCOPY)
template <typename T>
cudaError_t launch_avgrad_t(Ctx *c, int nvinv, int ncasc, T *grad, T *work, cudaStream_t st) {
  const size_t na35 = (size_t)c->rg.nnpinv * nvinv;
  for (int k = 0; k < ncasc; k++) {
    cudaError_t e = cudaMemcpyAsync(work, grad, sizeof(T) * na35, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    k_avgrad<T><<<(c->nnpg + 255) / 256, 256, 0, st>>>(c->nnpg, c->rg.ncon, nvinv, c->d_maskg,
                                                       c->d_mconn, c->d_ieng, grad, work);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = cudaMemcpyAsync(grad, work, sizeof(T) * na35, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_avgrad(Ctx *c, int nvinv, int ncasc, float *grad, cudaStream_t st) {
  return launch_avgrad_t<float>(c, nvinv, ncasc, grad, (float *)c->d_avg_work, st);
}

cudaError_t launch_avgrad8(Ctx *c, int nvinv, int ncasc, double *grad, cudaStream_t st) {
  return launch_avgrad_t<double>(c, nvinv, ncasc, grad, (double *)c->d_avg_work, st);
}

}  // namespace fem25
