// Exact adjoint gradient with respect to the anchor-node lambda, mu, rho:
//   g_{m,p} = sum_{pairs,s} Re( lam_s^H dA/dm_p u_s )
// evaluated without forming derivative matrices.  For the KM25ISOQ operator
// (estiff25.f:64-154) the bilinear form lam^H A u at a quadrature point with
// weight W = w_xi w_eta |J| splits into
//   lambda:  conj(div L) div U,   div V = V1,x + V3,z - i wpy V2
//   mu:      2 conj(L1,x) U1,x + 2 conj(L3,z) U3,z + 2 wpy^2 conj(L2) U2
//            + conj(L1,z + L3,x)(U1,z + U3,x)
//            + conj(L2,x - i wpy L1)(U2,x - i wpy U1)
//            + conj(L2,z - i wpy L3)(U2,z - i wpy U3)
//   rho:     -omega^2 sum_i conj(L_i) U_i
// and the derivative with respect to the anchor value m_p weights each point
// by the bilinear anchor function SF_p (cjac.f:98-108).  Fields are
// interpolated to the 13x13 points with the SHL table (dshl.f:1-243) and the
// inverse Jacobian (cjac.f:128-134).
#include <cstdlib>

#include "ctx.cuh"
#include "kcommon.cuh"

namespace fem25 {

constexpr int kGThreads = 192;   // >= 169 quadrature points
constexpr int kShlPad = (3 * kNq * kNen + 1) & ~1;  // shared SHL table, rounded to 16 B

struct GradArgs {
  int npairs, nsrc, ndof, nnpg;
  long long field_stride;  // complex entries per (pair, source) = ndof
};

__device__ __forceinline__ double re_cj(double ar, double ai, double br, double bi) {
  return ar * br + ai * bi;  // Re(conj(a) b)
}

// TILE sources of both fields are staged in shared memory per sync; the
// result does not depend on TILE (each point sums the sources in order).
template <int TILE>
__global__ void __launch_bounds__(kGThreads)
    k_grad_plain(MeshView mv, DevTables dt, GradArgs ga, const int *__restrict__ elems,
                 const int *__restrict__ lm, PairTable pt,
                 const double2 *__restrict__ u, const double2 *__restrict__ lam,
                 double *__restrict__ grad, int *__restrict__ err) {
  extern __shared__ double sm[];
  double *shl = sm;                                        // [169][25][3]
  // double2 staging area starts on a 16-byte boundary (12675 doubles -> 12676)
  double2 *fu = reinterpret_cast<double2 *>(sm + kShlPad);  // [tile][75]
  double2 *fl = fu + TILE * kNee;
  double *red = reinterpret_cast<double *>(fl + TILE * kNee);  // [12][kGThreads/32]
  const int t = threadIdx.x;
  for (int i = t; i < 3 * kNq * kNen; i += kGThreads) shl[i] = dt.shl[i];
  const int e = elems[blockIdx.x];
  const int4 ie = mv.ieng[e];
  const int *lme = lm + (size_t)e * kNee;
  // per-point geometry
  double ax = 0, bx = 0, az = 0, bz = 0, wq = 0;
  const bool act = t < kNq;
  if (act) {
    QGeo g;
    if (!quad_geo(mv, dt, ie, t, false, g)) atomicCAS(err, 0, e + 1);
    const int intx = t % kNint, intz = t / kNint;
    ax = g.dzdeta / g.rjac;
    bx = -g.dzdxi / g.rjac;
    az = -g.dxdeta / g.rjac;
    bz = g.dxdxi / g.rjac;
    wq = dt.wts[intx] * dt.wts[intz] * g.rjac;
  }
  double accl = 0.0, accm = 0.0, accr = 0.0;
  for (int p = 0; p < ga.npairs; p++) {
    const double2 pr = pt.p[p];
    const double w2 = pr.x * pr.x, wpy = pr.y;
    for (int s0 = 0; s0 < ga.nsrc; s0 += TILE) {
      const int ns = min(TILE, ga.nsrc - s0);
      __syncthreads();
      for (int i = t; i < ns * kNee; i += kGThreads) {
        const int s = i / kNee, k = i % kNee;
        const int d = lme[k];
        const size_t off = ((size_t)p * ga.nsrc + s0 + s) * ga.field_stride;
        fu[i] = d > 0 ? u[off + d - 1] : make_double2(0.0, 0.0);
        fl[i] = d > 0 ? lam[off + d - 1] : make_double2(0.0, 0.0);
      }
      __syncthreads();
      if (!act) continue;
      for (int s = 0; s < ns; s++) {
        double U[3][3][2], L[3][3][2];  // [comp][value, d/dxi, d/deta][re,im]
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
          for (int d = 0; d < 3; d++) U[k][d][0] = U[k][d][1] = L[k][d][0] = L[k][d][1] = 0.0;
        const double *sq = shl + 3 * kNen * t;
        const double2 *us = fu + s * kNee, *ls = fl + s * kNee;
#pragma unroll 5
        for (int a = 0; a < kNen; a++) {
          const double nxi = sq[3 * a], neta = sq[3 * a + 1], n = sq[3 * a + 2];
#pragma unroll
          for (int k = 0; k < 3; k++) {
            const double2 uv = us[3 * a + k], lv = ls[3 * a + k];
            U[k][0][0] += n * uv.x;    U[k][0][1] += n * uv.y;
            U[k][1][0] += nxi * uv.x;  U[k][1][1] += nxi * uv.y;
            U[k][2][0] += neta * uv.x; U[k][2][1] += neta * uv.y;
            L[k][0][0] += n * lv.x;    L[k][0][1] += n * lv.y;
            L[k][1][0] += nxi * lv.x;  L[k][1][1] += nxi * lv.y;
            L[k][2][0] += neta * lv.x; L[k][2][1] += neta * lv.y;
          }
        }
        // physical derivatives: d/dx = ax d/dxi + bx d/deta, d/dz = az d/dxi + bz d/deta
        double Ux[3][2], Uz[3][2], Lx[3][2], Lz[3][2];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
          for (int c = 0; c < 2; c++) {
            Ux[k][c] = ax * U[k][1][c] + bx * U[k][2][c];
            Uz[k][c] = az * U[k][1][c] + bz * U[k][2][c];
            Lx[k][c] = ax * L[k][1][c] + bx * L[k][2][c];
            Lz[k][c] = az * L[k][1][c] + bz * L[k][2][c];
          }
        // div V = V1,x + V3,z - i wpy V2
        const double du_r = Ux[0][0] + Uz[2][0] + wpy * U[1][0][1];
        const double du_i = Ux[0][1] + Uz[2][1] - wpy * U[1][0][0];
        const double dl_r = Lx[0][0] + Lz[2][0] + wpy * L[1][0][1];
        const double dl_i = Lx[0][1] + Lz[2][1] - wpy * L[1][0][0];
        accl += re_cj(dl_r, dl_i, du_r, du_i);
        double bm = 2.0 * re_cj(Lx[0][0], Lx[0][1], Ux[0][0], Ux[0][1]) +
                    2.0 * re_cj(Lz[2][0], Lz[2][1], Uz[2][0], Uz[2][1]) +
                    2.0 * wpy * wpy * re_cj(L[1][0][0], L[1][0][1], U[1][0][0], U[1][0][1]);
        bm += re_cj(Lz[0][0] + Lx[2][0], Lz[0][1] + Lx[2][1], Uz[0][0] + Ux[2][0],
                    Uz[0][1] + Ux[2][1]);
        // V2,x - i wpy V1
        bm += re_cj(Lx[1][0] + wpy * L[0][0][1], Lx[1][1] - wpy * L[0][0][0],
                    Ux[1][0] + wpy * U[0][0][1], Ux[1][1] - wpy * U[0][0][0]);
        // V2,z - i wpy V3
        bm += re_cj(Lz[1][0] + wpy * L[2][0][1], Lz[1][1] - wpy * L[2][0][0],
                    Uz[1][0] + wpy * U[2][0][1], Uz[1][1] - wpy * U[2][0][0]);
        accm += bm;
        double br = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) br += re_cj(L[k][0][0], L[k][0][1], U[k][0][0], U[k][0][1]);
        accr += -w2 * br;
      }
    }
  }
  // g_{m, anchor a} = sum_q SF_a(q) W_q acc_m(q)
  double v[12];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const double f = act ? dt.sf[4 * t + a] * wq : 0.0;
    v[3 * a + 0] = f * accl;
    v[3 * a + 1] = f * accm;
    v[3 * a + 2] = f * accr;
  }
#pragma unroll
  for (int k = 0; k < 12; k++) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    v[k] = x;
  }
  const int warp = t / 32, lane = t % 32, nw = kGThreads / 32;
  __syncthreads();
  if (lane == 0)
    for (int k = 0; k < 12; k++) red[k * nw + warp] = v[k];
  __syncthreads();
  if (t < 12) {
    double x = 0.0;
    for (int w = 0; w < nw; w++) x += red[t * nw + w];
    const int a = t / 3, m = t % 3;
    const int anchor = (a == 0 ? ie.x : a == 1 ? ie.y : a == 2 ? ie.z : ie.w) - 1;
    atomicAdd(&grad[(size_t)m * ga.nnpg + anchor], x);
  }
}

static size_t grad_smem(int tile) {
  return sizeof(double) * kShlPad + sizeof(double2) * 2 * tile * kNee +
         sizeof(double) * 12 * (kGThreads / 32);
}

template <int TILE>
static cudaError_t grad_tile_launch(Ctx *c, const GradArgs &ga, const PairTable &pt,
                                    const double *u, const double *lam, double *grad,
                                    cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_grad_plain<TILE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)grad_smem(TILE))))
    return e;
  k_grad_plain<TILE><<<c->n_nonpml, kGThreads, grad_smem(TILE), st>>>(
      c->mv, c->dt, ga, c->d_nonpml, c->d_lm, pt, (const double2 *)u, (const double2 *)lam, grad,
      c->d_err);
  return cudaGetLastError();
}

static const int kGradTiles[] = {2, 4, 8};

static cudaError_t grad_variant(Ctx *c, int tile, const GradArgs &ga, const PairTable &pt,
                                const double *u, const double *lam, double *grad,
                                cudaStream_t st) {
  switch (tile) {
    case 2: return grad_tile_launch<2>(c, ga, pt, u, lam, grad, st);
    case 8: return grad_tile_launch<8>(c, ga, pt, u, lam, grad, st);
    default: return grad_tile_launch<4>(c, ga, pt, u, lam, grad, st);
  }
}

// The source-tile width (sources of both fields staged per shared-memory
// pass: 2, 4 or 8, trading shared memory per CTA against syncs per source) is
// picked on the first call of a context by timing each width once on that
// call's fields into a scratch gradient, and kept.  FEM25_GRAD_TILE forces a
// width; a call recorded into a CUDA graph before any tuning uses 4.
cudaError_t launch_grad_plain(Ctx *c, const PairTable &pt, int npairs, int nsrc, const double *u,
                              const double *lam, double *grad, cudaStream_t st) {
  GradArgs ga;
  ga.npairs = npairs;
  ga.nsrc = nsrc;
  ga.ndof = c->ndof;
  ga.nnpg = c->nnpg;
  ga.field_stride = c->ndof;
  if (c->n_nonpml == 0) return cudaSuccess;
  cudaError_t e;
  if (c->grad_tile < 0) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    const char *env = std::getenv("FEM25_GRAD_TILE");
    if (env) {
      const int t = std::atoi(env);
      c->grad_tile = (t == 2 || t == 8) ? t : 4;
    } else if (cs != cudaStreamCaptureStatusNone) {
      c->grad_tile = 4;
    } else {
      double *scratch = nullptr;
      if ((e = cudaMalloc(&scratch, sizeof(double) * 3 * (size_t)c->nnpg))) return e;
      cudaEvent_t ev[4];
      for (auto &x : ev) cudaEventCreate(&x);
      cudaEventRecord(ev[0], st);
      for (int k = 0; k < 3; k++) {
        if ((e = grad_variant(c, kGradTiles[k], ga, pt, u, lam, scratch, st))) break;
        cudaEventRecord(ev[k + 1], st);
      }
      if (!e) e = cudaEventSynchronize(ev[3]);
      float best = 1e30f;
      for (int k = 0; k < 3 && !e; k++) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        if (t < best) {
          best = t;
          c->grad_tile = kGradTiles[k];
        }
      }
      for (auto &x : ev) cudaEventDestroy(x);
      cudaFree(scratch);
      if (e) return e;
    }
  }
  return grad_variant(c, c->grad_tile, ga, pt, u, lam, grad, st);
}

}  // namespace fem25
