// Exact lambda/mu/rho adjoint gradient with the interpolation on the 5th
// generation tensor cores in split precision (3xTF32, FP32 accumulation in
// TMEM), FP64 accumulation across (omega, py) pairs and sources.
//
// For an element e and a "combo" c = (pair p, source s) the forward and
// adjoint fields give 12 real nodal vectors (u and lambda, 3 components,
// real and imaginary part) of 25 values.  Their values and reference
// derivatives at the 13x13 quadrature points are a GEMM with the constant
// shape-function table (SHL, dshl.f:1-243) as the A operand:
//     D_d[q][c*12 + v] = sum_a SHL_d[q][a] * B[a][c*12 + v],   d = N, dN/dxi, dN/deta
// M = 169 points (two 128-row tiles), N = 128 columns (10 combos x 12
// vectors + 8 zero columns), K = 25 nodes (padded to 32).  One epilogue
// thread owns one quadrature point (one TMEM lane) and finds all 36 values
// of a combo in its own lane: it applies the inverse Jacobian (cjac.f:128-134)
// and forms the lambda, mu, rho bilinear forms of KM25ISOQ
// (estiff25.f:64-154), exactly as the FP64 kernel in k_grad.cu does.
//
// Split precision: x = hi + lo with hi = tf32(x), lo = tf32(x - hi) for both
// operands; D = A_hi B_hi + A_hi B_lo + A_lo B_hi (the A_lo B_lo term, ~2^-22
// relative, is dropped).  Operands are staged in shared memory in the
// SWIZZLE_NONE K-major canonical layout (8-row x 16-byte core matrices) and
// described with tcgen05 shared-memory descriptors; one elected thread issues
// the MMAs and commits to an mbarrier that the epilogue warps wait on with a
// bounded spin.
#include <cstdint>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "kcommon.cuh"

namespace fem25 {

namespace tc {
constexpr int kThreads = 256;             // 8 warps; warps 0-3 = epilogue (TMEM lanes 0-127)
constexpr int kCombos = 10;               // (pair, source) combos per MMA batch
constexpr int kN = 128;                   // MMA N: 10 x 12 vectors + 8 zero columns
constexpr int kK = 32;                    // 25 nodes + 7 zero rows
constexpr int kTileRows = 128;            // MMA M
constexpr int kTailRows = 48;             // rows stored for the second M tile (41 used)
// A tables: [d][hi/lo] full tile (128 rows), then [d][hi/lo] tail tile (48 rows)
constexpr int kAFullLbo = kTileRows / 8 * 128;   // 2048 B between K chunks
constexpr int kATailLbo = kTailRows / 8 * 128;   // 768 B
constexpr int kAFullBytes = kAFullLbo * (kK / 4);  // 16 KB
constexpr int kATailBytes = kATailLbo * (kK / 4);  // 6 KB
constexpr int kABytes = 3 * 2 * (kAFullBytes + kATailBytes);  // 132 KB
constexpr int kBLbo = kN / 8 * 128;                // 2048 B
constexpr int kBBytes = kBLbo * (kK / 4);          // 16 KB per hi/lo
constexpr int kSmemBytes = kABytes + 2 * kBBytes + 1024;  // + B slack read by the tail tile
constexpr uint32_t kTmemCols = 512;
constexpr long long kSpinLimit = 1LL << 26;
}  // namespace tc

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// tcgen05 shared-memory matrix descriptor, SWIZZLE_NONE, K-major
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                 // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor: D f32, A/B tf32, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(tc::kN >> 3) << 17) |
                            ((uint32_t)(tc::kTileRows >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// 16 consecutive TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// byte offset of element (row, k) in a K-major SWIZZLE_NONE tile with the
// given distance between K chunks (LBO); core matrices of 8 rows x 16 bytes
__host__ __device__ __forceinline__ uint32_t kmajor_off(int row, int k, uint32_t lbo) {
  return (uint32_t)((row >> 3) * 128 + (row & 7) * 16 + (k >> 2) * lbo + (k & 3) * 4);
}

struct TcArgs {
  int npairs, nsrc, ndof, nnpg, n_elem;
  long long ncombo;  // npairs * nsrc
};

__global__ void __launch_bounds__(tc::kThreads, 1)
    k_grad_tc(MeshView mv, DevTables dt, TcArgs ga, const int *__restrict__ elems,
              const int *__restrict__ lm, const double2 *__restrict__ pairs,
              const double2 *__restrict__ u, const double2 *__restrict__ lam,
              const uint8_t *__restrict__ atab, double *__restrict__ grad, int *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *sA = sm;                                  // constant SHL tables
  uint8_t *sB = sm + tc::kABytes;                    // [hi/lo][16 KB]
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int abort_s;
  __shared__ float2 cpar[tc::kCombos];               // (omega^2, omega*py) per combo slot
  __shared__ double red[12][8];
  __shared__ int lme[kNee];
  __shared__ int4 ie_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // ---- constant A tables and zeroed B padding
  for (int i = tid * 16; i < tc::kABytes; i += tc::kThreads * 16)
    *reinterpret_cast<uint4 *>(sA + i) = *reinterpret_cast<const uint4 *>(atab + i);
  for (int i = tid * 16; i < 2 * tc::kBBytes + 1024; i += tc::kThreads * 16)
    *reinterpret_cast<uint4 *>(sB + i) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    abort_s = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(tc::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const uint32_t mbar_a = smem_u32(&mbar);
  uint32_t phase = 0;

  const uint32_t sA_a = smem_u32(sA), sB_a = smem_u32(sB);

  for (int ei = blockIdx.x; ei < ga.n_elem; ei += gridDim.x) {
    const int e = elems[ei];
    if (tid < kNee) lme[tid] = lm[(size_t)e * kNee + tid];
    if (tid == 0) ie_s = mv.ieng[e];
    __syncthreads();
    // per-point geometry for the two points of this thread (epilogue warps)
    float gax[2] = {0, 0}, gbx[2] = {0, 0}, gaz[2] = {0, 0}, gbz[2] = {0, 0};
    double racc[2][3] = {{0, 0, 0}, {0, 0, 0}};
    if (warp < 4) {
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int q = t * tc::kTileRows + tid;
        if (q < kNq) {
          QGeo g;
          if (!quad_geo(mv, dt, ie_s, q, false, g)) atomicCAS(err, 0, e + 1);
          gax[t] = (float)(g.dzdeta / g.rjac);
          gbx[t] = (float)(-g.dzdxi / g.rjac);
          gaz[t] = (float)(-g.dxdeta / g.rjac);
          gbz[t] = (float)(g.dxdxi / g.rjac);
        }
      }
    }
    for (long long c0 = 0; c0 < ga.ncombo; c0 += tc::kCombos) {
      const int nc = (int)min((long long)tc::kCombos, ga.ncombo - c0);
      // ---- gather B: rows = combo*12 + vec, K = node; hi at sB, lo at sB + 16 KB
      if (tid < nc) {
        const double2 pr = pairs[(c0 + tid) / ga.nsrc];
        cpar[tid] = make_float2((float)(pr.x * pr.x), (float)pr.y);
      }
      for (int it = tid; it < nc * 2 * kNee; it += tc::kThreads) {
        const int cs = it / (2 * kNee), r = it % (2 * kNee);
        const int f = r / kNee, k = r % kNee;      // field (u / lambda), element equation
        const int a = k / 3, comp = k % 3;
        const int d = lme[k];
        double2 v = make_double2(0.0, 0.0);
        if (d > 0) {
          const size_t off = (size_t)(c0 + cs) * ga.ndof + d - 1;
          v = f == 0 ? u[off] : lam[off];
        }
        const int row = cs * 12 + f * 6 + comp * 2;
#pragma unroll
        for (int ri = 0; ri < 2; ri++) {
          const float x = (float)(ri == 0 ? v.x : v.y);
          const uint32_t hi = to_tf32(x);
          const uint32_t lo = to_tf32(x - __uint_as_float(hi));
          const uint32_t o = kmajor_off(row + ri, a, tc::kBLbo);
          *reinterpret_cast<uint32_t *>(sB + o) = hi;
          *reinterpret_cast<uint32_t *>(sB + tc::kBBytes + o) = lo;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      for (int mt = 0; mt < 2; mt++) {
        // ---- MMAs of this M tile: 3 tables x 4 K steps x 3 split terms
        if (tid == 128) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          for (int d = 0; d < 3; d++) {
            const uint32_t abase = sA_a + (mt == 0 ? (uint32_t)(d * 2) * tc::kAFullBytes
                                                   : (uint32_t)(6 * tc::kAFullBytes + d * 2 * tc::kATailBytes));
            const uint32_t alo = mt == 0 ? tc::kAFullBytes : tc::kATailBytes;
            const uint32_t albo = mt == 0 ? tc::kAFullLbo : tc::kATailLbo;
            const uint32_t td = tmem + (uint32_t)(d * tc::kN);
            for (int ks = 0; ks < tc::kK / 8; ks++) {
              const uint64_t ahi = umma_desc(abase + 2 * ks * albo, albo, 128);
              const uint64_t alo_d = umma_desc(abase + alo + 2 * ks * albo, albo, 128);
              const uint64_t bhi = umma_desc(sB_a + 2 * ks * tc::kBLbo, tc::kBLbo, 128);
              const uint64_t blo = umma_desc(sB_a + tc::kBBytes + 2 * ks * tc::kBLbo, tc::kBLbo, 128);
              mma_tf32(td, ahi, bhi, ks > 0 ? 1u : 0u);
              mma_tf32(td, ahi, blo, 1u);
              mma_tf32(td, alo_d, bhi, 1u);
            }
          }
          mma_commit(mbar_a);
        }
        // ---- epilogue: warps 0-3, one quadrature point per TMEM lane
        if (warp < 4) {
          long long spins = 0;
          while (!mbar_try_wait(mbar_a, phase)) {
            if (++spins > tc::kSpinLimit) {
              atomicCAS(err, 0, -1000000);
              abort_s = 1;
              break;
            }
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int q = mt * tc::kTileRows + tid;
          const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
          float tl = 0.f, tm = 0.f, tr = 0.f;
          for (int g0 = 0; g0 < nc; g0 += 4) {
            float vals[3][48];
            const int ncol = (g0 + 4 <= tc::kCombos) ? 48 : 32;  // last group: columns 96..127
#pragma unroll
            for (int d = 0; d < 3; d++) {
              tmem_ld16(lane_addr + (uint32_t)(d * tc::kN + g0 * 12), vals[d]);
              tmem_ld16(lane_addr + (uint32_t)(d * tc::kN + g0 * 12 + 16), vals[d] + 16);
              if (ncol == 48) tmem_ld16(lane_addr + (uint32_t)(d * tc::kN + g0 * 12 + 32), vals[d] + 32);
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (q < kNq) {
              const int t = mt;
#pragma unroll
              for (int cc = 0; cc < 4; cc++) {
                if (g0 + cc >= nc) break;
                const float w2 = cpar[g0 + cc].x, wpy = cpar[g0 + cc].y;
                // U[k][c]: value, Ux, Uz of field u (f=0) and lambda (f=1)
                float V[2][3][2], X[2][3][2], Z[2][3][2];
#pragma unroll
                for (int f = 0; f < 2; f++)
#pragma unroll
                  for (int k = 0; k < 3; k++)
#pragma unroll
                    for (int ri = 0; ri < 2; ri++) {
                      const int col = cc * 12 + f * 6 + k * 2 + ri;
                      const float val = vals[0][col], dxi = vals[1][col], deta = vals[2][col];
                      V[f][k][ri] = val;
                      X[f][k][ri] = gax[t] * dxi + gbx[t] * deta;
                      Z[f][k][ri] = gaz[t] * dxi + gbz[t] * deta;
                    }
                // div V = V1,x + V3,z - i wpy V2
                const float du_r = X[0][0][0] + Z[0][2][0] + wpy * V[0][1][1];
                const float du_i = X[0][0][1] + Z[0][2][1] - wpy * V[0][1][0];
                const float dl_r = X[1][0][0] + Z[1][2][0] + wpy * V[1][1][1];
                const float dl_i = X[1][0][1] + Z[1][2][1] - wpy * V[1][1][0];
                tl += dl_r * du_r + dl_i * du_i;
                float bm = 2.f * (X[1][0][0] * X[0][0][0] + X[1][0][1] * X[0][0][1]) +
                           2.f * (Z[1][2][0] * Z[0][2][0] + Z[1][2][1] * Z[0][2][1]) +
                           2.f * wpy * wpy * (V[1][1][0] * V[0][1][0] + V[1][1][1] * V[0][1][1]);
                bm += (Z[1][0][0] + X[1][2][0]) * (Z[0][0][0] + X[0][2][0]) +
                      (Z[1][0][1] + X[1][2][1]) * (Z[0][0][1] + X[0][2][1]);
                bm += (X[1][1][0] + wpy * V[1][0][1]) * (X[0][1][0] + wpy * V[0][0][1]) +
                      (X[1][1][1] - wpy * V[1][0][0]) * (X[0][1][1] - wpy * V[0][0][0]);
                bm += (Z[1][1][0] + wpy * V[1][2][1]) * (Z[0][1][0] + wpy * V[0][2][1]) +
                      (Z[1][1][1] - wpy * V[1][2][0]) * (Z[0][1][1] - wpy * V[0][2][0]);
                tm += bm;
                float br = 0.f;
#pragma unroll
                for (int k = 0; k < 3; k++) br += V[1][k][0] * V[0][k][0] + V[1][k][1] * V[0][k][1];
                tr += -w2 * br;
              }
            }
          }
          racc[mt][0] += (double)tl;
          racc[mt][1] += (double)tm;
          racc[mt][2] += (double)tr;
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        }
        phase ^= 1u;
        __syncthreads();
        if (abort_s) break;
      }
      if (abort_s) break;
    }
    // ---- g_{m, anchor a} += sum_q SF_a(q) W_q racc_m(q)
    double v[12];
#pragma unroll
    for (int k = 0; k < 12; k++) v[k] = 0.0;
    if (warp < 4) {
#pragma unroll
      for (int t = 0; t < 2; t++) {
        const int q = t * tc::kTileRows + tid;
        if (q < kNq) {
          const int intx = q % kNint, intz = q / kNint;
          QGeo g;
          quad_geo(mv, dt, ie_s, q, false, g);
          const double wq = dt.wts[intx] * dt.wts[intz] * g.rjac;
#pragma unroll
          for (int a = 0; a < 4; a++) {
            const double fw = dt.sf[4 * q + a] * wq;
            v[3 * a + 0] += fw * racc[t][0];
            v[3 * a + 1] += fw * racc[t][1];
            v[3 * a + 2] += fw * racc[t][2];
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double x = v[k];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      v[k] = x;
    }
    if (lane == 0)
      for (int k = 0; k < 12; k++) red[k][warp] = v[k];
    __syncthreads();
    if (tid < 12) {
      double x = 0.0;
      for (int w = 0; w < 4; w++) x += red[tid][w];
      const int a = tid / 3, m = tid % 3;
      const int anchor = (a == 0 ? ie_s.x : a == 1 ? ie_s.y : a == 2 ? ie_s.z : ie_s.w) - 1;
      atomicAdd(&grad[(size_t)m * ga.nnpg + anchor], x);
    }
    __syncthreads();
    if (abort_s) break;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kTmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// host: A tables (SHL in tf32 hi/lo, K-major canonical layout)
// ---------------------------------------------------------------------------
static uint32_t host_tf32(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7f800000u) == 0x7f800000u) return b & 0xffffe000u;
  b += 0x1000u;  // round half away from zero on the 13 dropped bits
  return b & 0xffffe000u;
}

std::vector<uint8_t> build_tc_tables(const Tables &t) {
  std::vector<uint8_t> buf(tc::kABytes, 0);
  auto put = [&](size_t off, uint32_t v) { std::memcpy(&buf[off], &v, 4); };
  for (int d = 0; d < 3; d++) {
    const int comp = d == 0 ? 2 : d - 1;  // SHL(3,...) = N, SHL(1,...) = dN/dxi, SHL(2,...) = dN/deta
    for (int q = 0; q < kNq; q++)
      for (int a = 0; a < kNen; a++) {
        const double x = t.shl[3 * ((size_t)a + (size_t)kNen * q) + comp];
        const float xf = (float)x;
        const uint32_t hi = host_tf32(xf);
        float hif;
        std::memcpy(&hif, &hi, 4);
        const uint32_t lo = host_tf32(xf - hif);
        if (q < tc::kTileRows) {
          const size_t base = (size_t)d * 2 * tc::kAFullBytes;
          put(base + kmajor_off(q, a, tc::kAFullLbo), hi);
          put(base + tc::kAFullBytes + kmajor_off(q, a, tc::kAFullLbo), lo);
        } else {
          const size_t base = (size_t)6 * tc::kAFullBytes + (size_t)d * 2 * tc::kATailBytes;
          const int r = q - tc::kTileRows;
          put(base + kmajor_off(r, a, tc::kATailLbo), hi);
          put(base + tc::kATailBytes + kmajor_off(r, a, tc::kATailLbo), lo);
        }
      }
  }
  return buf;
}

cudaError_t launch_grad_tc(Ctx *c, int npairs, int nsrc, const double *u, const double *lam,
                           double *grad, cudaStream_t st) {
  cudaError_t e;
  if (!c->d_tc_tab) {
    std::vector<uint8_t> h = build_tc_tables(c->tab);
    if ((e = cudaMalloc(&c->d_tc_tab, h.size()))) return e;
    if ((e = cudaMemcpy(c->d_tc_tab, h.data(), h.size(), cudaMemcpyHostToDevice))) return e;
    if ((e = cudaFuncSetAttribute(k_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  tc::kSmemBytes)))
      return e;
  }
  if (c->n_nonpml == 0) return cudaSuccess;
  TcArgs ga;
  ga.npairs = npairs;
  ga.nsrc = nsrc;
  ga.ndof = c->ndof;
  ga.nnpg = c->nnpg;
  ga.n_elem = c->n_nonpml;
  ga.ncombo = (long long)npairs * nsrc;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int grid = std::min(nsm, c->n_nonpml);
  k_grad_tc<<<grid, tc::kThreads, tc::kSmemBytes, st>>>(c->mv, c->dt, ga, c->d_nonpml, c->d_lm,
                                                         c->d_pairs, (const double2 *)u,
                                                         (const double2 *)lam, c->d_tc_tab, grad,
                                                         c->d_err);
  return cudaGetLastError();
}

}  // namespace fem25
