// Exact lambda/mu/rho adjoint gradient with the interpolation on the 5th
// generation tensor cores in split precision (3xTF32, FP32 accumulation in
// TMEM), FP64 accumulation across (omega, py) pairs and sources.
//
// For an element e and a "combo" c = (pair p, source s) the forward and
// adjoint fields give 12 real nodal vectors (u and lambda, 3 components,
// real and imaginary part) of 25 values.  Their values and reference
// derivatives at the 13x13 quadrature points are a GEMM with the constant
// shape-function table (SHL, dshl.f:1-243) as the A operand:
//     D[(d, q)][c*12 + v] = sum_a SHL_d[q][a] * B[c*12 + v][a],   d = N, dN/dxi, dN/deta
// The 3 x 169 = 507 rows (d, q) are cut into four 128-row chains:
//     chain 0, 1, 2: d = N, dN/dxi, dN/deta at q = 0..127 (TMEM lane = q)
//     chain 3:       the 41 points q = 128..168, three adjacent lanes per
//                    point (lane 32w + 3j + d for q = 128 + 10w + j, j < 10);
//                    the last point uses lanes 30, 31 and 62
// so one thread of chains 0-2 finds the 36 values of a combo at its point in
// its own TMEM lane.  A chain-3 warp copies its TMEM rows into a shared-
// memory area private to the warp (point 168's rows, which span two warps,
// into a shared buffer) and releases TMEM at once; the three lanes of a point
// then compute combos t and t+3.  N = 64 columns = 5 combos x 12 vectors + 4
// zero columns.  Each point's values then get the inverse
// Jacobian (cjac.f:128-134) and the lambda, mu, rho bilinear forms of
// KM25ISOQ (estiff25.f:64-154), as in the FP64 kernel of k_grad.cu,
// accumulated per point in FP64.
//
// Split precision: x = hi + lo with hi = tf32(x), lo = tf32(x - hi) for both
// operands; D = A_hi B_hi + A_hi B_lo + A_lo B_hi (the A_lo B_lo term, ~2^-22
// relative, is dropped).  Fields enter centred: node column a holds the
// node's deviation from the element's centre node (an FP64 difference) and
// column 25 the centre value, which the tables weight by 1 in the value rows
// and 0 in the derivative rows, so derivatives of smooth fields are formed
// from the small deviations without cancellation.
// With K segments of 28 columns (25 nodes, the centre value, 2 zero):
//     A' = [A_hi | A_lo]                (56 columns, 7 MMA K-steps)
//     B1 = [B_hi | B_hi],  B2 = [B_lo | 4 zero columns]
//     D  = A' B1  (A_hi B_hi + A_lo B_hi)  +  A'[:, 0:32] B2  (A_hi B_lo)
// 11 K-steps in all; the second product reuses the A_hi chunks (its last
// chunk reaches 4 A_lo columns, multiplied by B2's zero columns).  Operands
// are staged in shared memory in the SWIZZLE_NONE K-major canonical layout
// (8-row x 16-byte core matrices) and described with tcgen05 shared-memory
// descriptors; with N = 64 the MMAs are bound by the shared-memory operand
// reads (about 128 B per clock), so A is kept small.
//
// One persistent CTA per SM, warp-specialised and pipelined over "stages"
// (element, batch of 5 combos):
//   warps 13-15  producers: gather the stage's nodal values (FP64 -> tf32
//                hi/lo) into one of 3 shared-memory B buffers
//   warp 12      MMA issuer (one thread): 4 chains x 11 K-steps
//                into one of 2 TMEM accumulator stages (2 x 256 columns)
//   warps 0-7    epilogue of chains 0-2 (warp w: lanes 32(w%4).., combos
//                {0,1,2} for w < 4, {3,4} otherwise)
//   warps 8-11   epilogue of chain 3
// Hand-offs are mbarriers; every wait is bounded (about half a second of SM
// clock).  A wait that runs out sets the context's error word and puts the
// CTA in a drain mode that runs the remaining schedule without waiting, so
// every named barrier is still reached; the MMA thread waits (bounded) for
// its MMAs and TMEM is freed before the CTA exits.
#include <cstdint>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "kcommon.cuh"
#include "tcgen05.cuh"

namespace fem25 {

namespace tc {
constexpr int kThreads = 512;
constexpr int kTailWarp0 = 8;        // warps 8-11
constexpr int kMmaWarp = 12;
constexpr int kProdWarp0 = 13;       // warps 13-15
constexpr int kProdThreads = 96;
constexpr int kEpiThreads = 384;     // warps 0-11
constexpr int kC = 5;                // combos per stage
constexpr int kN = 64;               // MMA N
constexpr int kSeg = 28;             // K segment: 25 nodes + 3 zero columns (7 chunks)
constexpr int kACols = 2 * kSeg;     // A' = [A_hi | A_lo]
constexpr int kB1Cols = 2 * kSeg;    // B1 = [B_hi | B_hi]
constexpr int kB2Cols = 32;          // B2 = [B_lo | 0]
constexpr int kSteps1 = kACols / 8;  // 7 K-steps of A' B1
constexpr int kSteps2 = kB2Cols / 8; // 4 K-steps of A'[:, 0:32] B2
constexpr int kTail = kNq - 128;     // 41 points in chain 3
constexpr int kALbo = 128 / 8 * 128;             // 2048 B between K chunks of A
constexpr int kAChain = kALbo * (kACols / 4);    // 28 KB per chain
constexpr int kABytes = 4 * kAChain;             // 112 KB
constexpr int kBLbo = kN / 8 * 128;              // 1024 B
constexpr int kBStage = kBLbo * ((kB1Cols + kB2Cols) / 4);  // 22 KB: B1 then B2
constexpr int kNB = 3;                           // B buffers
constexpr int kStgStride = 61;                   // chain-3 staging row: 5 combos + 1 pad
constexpr int kStgRows = 32;                     // one row per lane
constexpr int kStgBytes = 4 * kStgRows * kStgStride * 4;
constexpr int kSmemBytes = kABytes + kNB * kBStage + kStgBytes;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kTmemStage = 256;
constexpr int kRefNode = 12;                     // centre node: reference of the deviations
constexpr int kRefCol = 25;                      // K column of the reference values
constexpr int kNodeItems = 3;                    // gather items (nodes) per producer thread
constexpr int kItemSlots = kProdThreads * kNodeItems;  // 288 slots for 250 items
constexpr int kTabBytes = kABytes + kItemSlots * 4;    // A tables + slot -> item map
static_assert(kItemSlots >= kC * 2 * kNen, "producer coverage");
static_assert(kTail == 41 && kC * 12 <= kN, "chain layout");
}  // namespace tc

// instruction descriptor: D f32, A/B tf32, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = tf32_idesc(128, tc::kN);

// TMEM lane of row (table d, tail point qt) in chain 3
__host__ __device__ __forceinline__ int tail_lane(int d, int qt) {
  if (qt < 40) return 32 * (qt / 10) + 3 * (qt % 10) + d;
  return d == 0 ? 30 : d == 1 ? 31 : 62;
}

struct TcArgs {
  int npairs, nsrc, ndof, nnpg, n_elem;
  int ncombo;      // npairs * nsrc
  int inject;      // 1: the first producer warp of CTA 0 withholds its first
                   // stage arrival, so the MMA thread's wait runs out (a test
                   // of the time-out path)
  long long spin;  // SM clocks a pipeline wait may take before it gives up
};

// Per-point geometry of the epilogue: inverse-Jacobian rows and W_q SF_a(q).
struct PointGeo {
  float ax, bx, az, bz;
  double wsf[4];
};

__device__ __forceinline__ void point_geo(const MeshView &mv, const DevTables &dt, int4 ie, int q,
                                          int e, int *err, PointGeo &pg) {
  QGeo g;
  if (!quad_geo(mv, dt, ie, q, false, g)) atomicCAS(err, 0, e + 1);
  pg.ax = (float)(g.dzdeta / g.rjac);
  pg.bx = (float)(-g.dzdxi / g.rjac);
  pg.az = (float)(-g.dxdeta / g.rjac);
  pg.bz = (float)(g.dxdxi / g.rjac);
  const double wq = dt.wts[q % kNint] * dt.wts[q / kNint] * g.rjac;
#pragma unroll
  for (int a = 0; a < 4; a++) pg.wsf[a] = dt.sf[4 * q + a] * wq;
}

// lambda, mu, rho forms of one combo at one point from its 36 interpolated
// values val[table][vector] (table: N, d/dxi, d/deta; vector: f*6 + k*2 + ri)
__device__ __forceinline__ void point_forms(const PointGeo &pg, float w2, float wpy,
                                            const float (*val)[12], float &tl, float &tm,
                                            float &tr) {
  float V[2][3][2], X[2][3][2], Z[2][3][2];
#pragma unroll
  for (int f = 0; f < 2; f++)
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
      for (int ri = 0; ri < 2; ri++) {
        const int v = f * 6 + k * 2 + ri;
        const float dxi = val[1][v], deta = val[2][v];
        V[f][k][ri] = val[0][v];
        X[f][k][ri] = pg.ax * dxi + pg.bx * deta;
        Z[f][k][ri] = pg.az * dxi + pg.bz * deta;
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
  // V2,x - i wpy V1
  bm += (X[1][1][0] + wpy * V[1][0][1]) * (X[0][1][0] + wpy * V[0][0][1]) +
        (X[1][1][1] - wpy * V[1][0][0]) * (X[0][1][1] - wpy * V[0][0][0]);
  // V2,z - i wpy V3
  bm += (Z[1][1][0] + wpy * V[1][2][1]) * (Z[0][1][0] + wpy * V[0][2][1]) +
        (Z[1][1][1] - wpy * V[1][2][0]) * (Z[0][1][1] - wpy * V[0][2][0]);
  tm += bm;
  float br = 0.f;
#pragma unroll
  for (int k = 0; k < 3; k++) br += V[1][k][0] * V[0][k][0] + V[1][k][1] * V[0][k][1];
  tr += -w2 * br;
}

__global__ void __launch_bounds__(tc::kThreads, 1)
    k_grad_tc(MeshView mv, DevTables dt, TcArgs ga, const int *__restrict__ elems,
              const int *__restrict__ lm, PairTable pt,
              const double2 *__restrict__ u, const double2 *__restrict__ lam,
              const uint8_t *__restrict__ atab, double *__restrict__ grad, int *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *sA = sm;                                        // 4 chains x (hi, lo)
  uint8_t *sB = sm + tc::kABytes;                          // kNB packed B tiles
  float *stg_all = reinterpret_cast<float *>(sm + tc::kABytes + tc::kNB * tc::kBStage);
  __shared__ uint64_t bar_bfull[tc::kNB], bar_bempty[tc::kNB], bar_tfull[2], bar_tempty[2];
  __shared__ uint64_t bar_drain;
  __shared__ uint32_t tmem_base_s;
  __shared__ int drain_s;
  __shared__ double red[12][12];
  __shared__ float p168[2][3][tc::kC * 12];  // point 168's rows: [stage parity][table][combo*12 + v]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int *drain = &drain_s;

  // ---- set-up: constant A tables, zeroed B buffers, barriers, TMEM
  for (int i = tid * 16; i < tc::kABytes; i += tc::kThreads * 16)
    *reinterpret_cast<uint4 *>(sA + i) = *reinterpret_cast<const uint4 *>(atab + i);
  for (int i = tid * 16; i < tc::kNB * tc::kBStage; i += tc::kThreads * 16)
    *reinterpret_cast<uint4 *>(sB + i) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    drain_s = 0;
    for (int b = 0; b < tc::kNB; b++) {
      mbar_init(smem_u32(&bar_bfull[b]), tc::kProdThreads / 32);  // one arrival per warp
      mbar_init(smem_u32(&bar_bempty[b]), 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(smem_u32(&bar_tfull[b]), 1);
      mbar_init(smem_u32(&bar_tempty[b]), tc::kEpiThreads / 32);
    }
    mbar_init(smem_u32(&bar_drain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == tc::kMmaWarp) {
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
  const int nb = (ga.ncombo + tc::kC - 1) / tc::kC;  // stages per element

  if (warp >= tc::kProdWarp0) {
    // =================== producers: nodal values -> tf32 hi/lo B tiles
    // Item j of this thread is (combo c, field f, node a) with
    // pt + 96 j = c*50 + f*25 + a, the same in every stage: the node's three
    // DOFs are consecutive (GENID numbers and fixes them together), so the
    // item is three adjacent complex values.  Loads are issued
    // unconditionally (inactive items read entries 0-2 and become zero) right
    // after the previous stage is stored, so they are in flight while the
    // producer waits for the next free buffer.
    // The slot -> item map (built on the host) gives the 32 lanes of each
    // store instruction items of different (row mod 8, column mod 4), the
    // shared-memory bank of a K-major core matrix, so the B' stores are about
    // 2-way instead of 8-way bank-conflicted.
    const int pt = tid - tc::kProdWarp0 * 32;
    const int *slot_item = reinterpret_cast<const int *>(atab + tc::kABytes);
    int meta[tc::kNodeItems];  // combo (bits 0-2), field (bit 3), node (bits 4-8); -1: none
#pragma unroll
    for (int j = 0; j < tc::kNodeItems; j++) {
      const int it = __ldg(slot_item + pt + j * tc::kProdThreads);
      const int r = it % (2 * kNen);
      meta[j] = it < 0 ? -1 : (it / (2 * kNen)) | ((r / kNen) << 3) | ((r % kNen) << 4);
    }
    if (blockIdx.x < ga.n_elem) {
      int dn[tc::kNodeItems];        // first DOF of the item's node (0: fixed)
      int dref = 0;                  // first DOF of the element's centre node
      double2 vn[tc::kNodeItems][3];  // the stage being gathered
      double2 rn[tc::kNodeItems][3];  // its centre-node values (same combo and field)
      int ei = blockIdx.x, b = 0;
#define FEM25_TC_LOAD_DOFS(EI)                                                   \
  do {                                                                            \
    const int e_ = elems[EI];                                                     \
    _Pragma("unroll") for (int j = 0; j < tc::kNodeItems; j++) dn[j] =            \
        meta[j] < 0 ? 0 : __ldg(lm + (size_t)e_ * kNee + 3 * (meta[j] >> 4));     \
    dref = __ldg(lm + (size_t)e_ * kNee + 3 * tc::kRefNode);                      \
  } while (0)
#define FEM25_TC_LOAD_STAGE(B)                                                   \
  do {                                                                            \
    const int c0_ = (B) * tc::kC;                                                 \
    const int nitems_ = min(tc::kC, ga.ncombo - c0_) * 2 * kNen;                  \
    const double2 *ub_ = u + (size_t)c0_ * ga.ndof, *lb_ = lam + (size_t)c0_ * ga.ndof; \
    _Pragma("unroll") for (int j = 0; j < tc::kNodeItems; j++) {                  \
      const bool cact_ = meta[j] >= 0 && (meta[j] & 7) < nitems_ / (2 * kNen);    \
      const bool act_ = cact_ && dn[j] > 0, ract_ = cact_ && dref > 0;            \
      const int off_ = act_ ? (meta[j] & 7) * ga.ndof + dn[j] - 1 : 0;            \
      const int roff_ = ract_ ? (meta[j] & 7) * ga.ndof + dref - 1 : 0;           \
      const double2 *p_ = ((meta[j] & 8) ? lb_ : ub_) + off_;                     \
      const double2 *q_ = ((meta[j] & 8) ? lb_ : ub_) + roff_;                    \
      _Pragma("unroll") for (int i = 0; i < 3; i++) {                             \
        const double2 x_ = __ldg(p_ + i), r_ = __ldg(q_ + i);                     \
        vn[j][i] = act_ ? x_ : make_double2(0.0, 0.0);                            \
        rn[j][i] = ract_ ? r_ : make_double2(0.0, 0.0);                           \
      }                                                                           \
    }                                                                             \
  } while (0)
      FEM25_TC_LOAD_DOFS(ei);
      FEM25_TC_LOAD_STAGE(0);
      for (uint32_t s = 0;; s++) {
        const int bs = (int)(s % tc::kNB);
        mbar_wait(smem_u32(&bar_bempty[bs]), ((s / tc::kNB) & 1u) ^ 1u, drain, err, -1000001,
                  ga.spin);
        uint8_t *bh = sB + bs * tc::kBStage;
        // items past the last combo of the stage store zeros into rows the
        // epilogue ignores; empty slots store nothing.  Centring: a node
        // column holds the node's deviation from the element's centre node
        // (FP64 difference), and column 25 the centre node's value itself,
        // which the A tables weight by 1 in the value rows and by 0 in the
        // derivative rows -- so derivatives are formed from the deviations
        // alone (smooth fields lose no digits to cancellation) and values
        // are centre + interpolated deviation.
#pragma unroll
        for (int j = 0; j < tc::kNodeItems; j++) {
          if (meta[j] >= 0) {
            const int row0 = (meta[j] & 7) * 12 + ((meta[j] >> 3) & 1) * 6, a = meta[j] >> 4;
            const double2 *rv = rn[j];  // centre values, gathered with the stage
            // B1 columns a and 28 + a hold hi, B2 column a (virtual column
            // 56 + a of the stage) holds lo
            const uint32_t o0 = kmajor_off(row0, a, tc::kBLbo);
            const uint32_t o1 = kmajor_off(row0, a + tc::kSeg, tc::kBLbo);
            const uint32_t o2 = kmajor_off(row0, a + tc::kB1Cols, tc::kBLbo);
            const uint32_t r0 = kmajor_off(row0, tc::kRefCol, tc::kBLbo);
            const uint32_t r1 = kmajor_off(row0, tc::kRefCol + tc::kSeg, tc::kBLbo);
            const uint32_t r2 = kmajor_off(row0, tc::kRefCol + tc::kB1Cols, tc::kBLbo);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
              for (int ri = 0; ri < 2; ri++) {
                // row0 is a multiple of 6 and the 6 rows of the node share one
                // 8-row core group only when row0 % 8 <= 2; the row offset is
                // recomputed per row
                const int row = row0 + 2 * i + ri;
                const uint32_t dr = (uint32_t)(((row >> 3) - (row0 >> 3)) * 128 + ((row & 7) - (row0 & 7)) * 16);
                const double rx = ri == 0 ? rv[i].x : rv[i].y;
                const float x = (float)((ri == 0 ? vn[j][i].x : vn[j][i].y) - rx);
                // hi: x rounded to 10 mantissa bits on the bit pattern; lo =
                // x - hi exactly, of which the MMA reads the top 19 bits
                const uint32_t hi = (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
                const uint32_t lo = __float_as_uint(x - __uint_as_float(hi));
                *reinterpret_cast<uint32_t *>(bh + o0 + dr) = hi;
                *reinterpret_cast<uint32_t *>(bh + o1 + dr) = hi;
                *reinterpret_cast<uint32_t *>(bh + o2 + dr) = lo;
                if (a == tc::kRefNode) {
                  const float xr = (float)rx;
                  const uint32_t hr = (__float_as_uint(xr) + 0x1000u) & 0xFFFFE000u;
                  const uint32_t lr = __float_as_uint(xr - __uint_as_float(hr));
                  *reinterpret_cast<uint32_t *>(bh + r0 + dr) = hr;
                  *reinterpret_cast<uint32_t *>(bh + r1 + dr) = hr;
                  *reinterpret_cast<uint32_t *>(bh + r2 + dr) = lr;
                }
              }
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        const bool withhold = ga.inject && blockIdx.x == 0 && warp == tc::kProdWarp0 && s == 0;
        if (lane == 0 && !withhold) mbar_arrive(smem_u32(&bar_bfull[bs]));
        int ein = ei, bn = b + 1;
        if (bn == nb) {
          bn = 0;
          ein += gridDim.x;
        }
        if (ein >= ga.n_elem) break;
        if (ein != ei) FEM25_TC_LOAD_DOFS(ein);
        FEM25_TC_LOAD_STAGE(bn);
        ei = ein;
        b = bn;
      }
#undef FEM25_TC_LOAD_DOFS
#undef FEM25_TC_LOAD_STAGE
    }
  } else if (warp == tc::kMmaWarp) {
    // =================== MMA issuer
    if (lane == 0) {
      // descriptors differ only in their start-address field (address >> 4,
      // below 2^14 for any shared-memory address), so offsets are added to a
      // base descriptor
      const uint64_t adesc = umma_desc(smem_u32(sA), tc::kALbo, 128);
      const uint64_t bdesc = umma_desc(smem_u32(sB), tc::kBLbo, 128);
      uint32_t s = 0;
      for (int ei = blockIdx.x; ei < ga.n_elem; ei += gridDim.x) {
        for (int b = 0; b < nb; b++, s++) {
          const int bs = (int)(s % tc::kNB), ts = (int)(s & 1u);
          mbar_wait(smem_u32(&bar_bfull[bs]), (s / tc::kNB) & 1u, drain, err, -1000002, ga.spin);
          mbar_wait(smem_u32(&bar_tempty[ts]), ((s >> 1) & 1u) ^ 1u, drain, err, -1000003,
                    ga.spin);
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint64_t bstage = bdesc + (uint64_t)((bs * tc::kBStage) >> 4);
          const uint32_t tstage = tmem + (uint32_t)(ts * tc::kTmemStage);
#pragma unroll 1
          for (int ch = 0; ch < 4; ch++) {
            const uint64_t achain = adesc + (uint64_t)((ch * tc::kAChain) >> 4);
            const uint32_t td = tstage + (uint32_t)(ch * tc::kN);
            // A' B1: A_hi B_hi + A_lo B_hi
#pragma unroll
            for (int ks = 0; ks < tc::kSteps1; ks++) {
              const uint64_t a = achain + (uint64_t)((2 * ks * tc::kALbo) >> 4);
              const uint64_t bd = bstage + (uint64_t)((2 * ks * tc::kBLbo) >> 4);
              mma_tf32(td, a, bd, kIdesc, ks > 0 ? 1u : 0u);
            }
            // A'[:, 0:32] B2: A_hi B_lo
#pragma unroll
            for (int ks = 0; ks < tc::kSteps2; ks++) {
              const uint64_t a = achain + (uint64_t)((2 * ks * tc::kALbo) >> 4);
              const uint64_t bd = bstage + (uint64_t)(((tc::kB1Cols / 4 + 2 * ks) * tc::kBLbo) >> 4);
              mma_tf32(td, a, bd, kIdesc, 1u);
            }
          }
          mma_commit(smem_u32(&bar_bempty[bs]));
          mma_commit(smem_u32(&bar_tfull[ts]));
        }
      }
      // every MMA issued above has completed once this commit arrives
      mma_commit(smem_u32(&bar_drain));
      const long long t0 = clock64();
      while (!mbar_try_wait(smem_u32(&bar_drain), 0u)) {
        if (clock64() - t0 > kTcSpinCycles) {
          atomicCAS(err, 0, -1000004);
          break;
        }
      }
    }
    __syncwarp();
  } else {
    // =================== epilogue (warps 0-11)
    const bool tail = warp >= tc::kTailWarp0;
    const int quarter = warp & 3;
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    // chain 0-2 threads: point q = lane index, combos {0,1,2} (warps 0-3) or {3,4}
    // chain 3 threads: lane 3j + t of quarter w holds table t of point
    // 128 + 10w + j and computes combo t of each round; point 168 has its
    // tables in lanes 30, 31 of quarter 0 and lane 30 of quarter 1 (xt)
    const int tt = quarter * 32 + lane;
    int q = tt, xt = -1;
    if (tail) {
      q = lane < 30 ? 128 + 10 * quarter + lane / 3 : -1;
      if (quarter == 0 && lane >= 30) xt = lane - 30;
      if (quarter == 1 && lane == 30) xt = 2;
      if (xt >= 0) q = 168;
    }
    const int tsel = lane % 3;
    const int cfirst = warp < 4 ? 0 : 3;
    const int clast = warp < 4 ? 2 : tc::kC - 1;
    uint32_t rnd = 0;  // stages so far (parity picks the p168 buffer)
    uint32_t s = 0;
    for (int ei = blockIdx.x; ei < ga.n_elem; ei += gridDim.x) {
      const int e = elems[ei];
      const int4 ie = mv.ieng[e];
      PointGeo pg;
      pg.ax = pg.bx = pg.az = pg.bz = 0.f;
#pragma unroll
      for (int a = 0; a < 4; a++) pg.wsf[a] = 0.0;
      if (q >= 0) point_geo(mv, dt, ie, q, e, err, pg);
      double racc[3] = {0.0, 0.0, 0.0};
      for (int b = 0; b < nb; b++, s++) {
        const int ts = (int)(s & 1u);
        const int c0 = b * tc::kC;
        const int nc = min(tc::kC, ga.ncombo - c0);
        mbar_wait(smem_u32(&bar_tfull[ts]), (s >> 1) & 1u, drain, err, -1000005, ga.spin);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tbase = tmem + lane_base + (uint32_t)(ts * tc::kTmemStage);
        float tl = 0.f, tm = 0.f, tr = 0.f;
        if (!tail) {
          const int cend = min(clast, nc - 1);
          if (cend < cfirst) {
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[ts]));
          }
          for (int c = cfirst; c <= cend; c++) {
            __syncwarp();
            float val[3][12];
#pragma unroll
            for (int d = 0; d < 3; d++)
#pragma unroll
              for (int j = 0; j < 3; j++)
                tmem_ld4(tbase + (uint32_t)(d * tc::kN + c * 12 + 4 * j), &val[d][4 * j]);
            tmem_wait_ld();
            if (c == cend) {
              asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
              __syncwarp();
              if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[ts]));
            }
            const double2 pr = pt.p[(c0 + c) / ga.nsrc];
            point_forms(pg, (float)(pr.x * pr.x), (float)pr.y, val, tl, tm, tr);
          }
        } else {
          // chain 3: this warp's TMEM rows -> its staging rows (row = lane),
          // point 168's rows -> p168 (double-buffered by stage parity so the
          // barrier of the next stage orders every reuse); TMEM is released
          // right after the copy
          float *stg = stg_all + quarter * tc::kStgRows * tc::kStgStride;
          const int rb = (int)(rnd++ & 1u);
          __syncwarp();
          {
            float *row = xt >= 0 ? &p168[rb][xt][0] : stg + lane * tc::kStgStride;
#pragma unroll
            for (int h = 0; h < 4; h++) {
              uint32_t r[16];
              tmem_ld16(tbase + (uint32_t)(3 * tc::kN + 16 * h), r);
              tmem_wait_ld();
#pragma unroll
              for (int k = 0; k < 16; k++)
                if (16 * h + k < 12 * nc) row[16 * h + k] = __uint_as_float(r[k]);
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[ts]));
          __syncwarp();
          if (quarter < 2) named_bar(3, 64);  // point 168's rows visible
          const int j3 = min(lane / 3, 9);  // lanes 30, 31 (no point of their own) read rows 27-29
#pragma unroll
          for (int rr = 0; rr < 2; rr++) {
            // unit of this lane: (point, combo t + 3 rr); rows of its three tables
            const int cl = (xt >= 0 ? xt : tsel) + 3 * rr;
            const float *r0, *r1, *r2;
            if (xt >= 0) {
              r0 = &p168[rb][0][0];
              r1 = &p168[rb][1][0];
              r2 = &p168[rb][2][0];
            } else {
              r0 = stg + (3 * j3) * tc::kStgStride;
              r1 = r0 + tc::kStgStride;
              r2 = r1 + tc::kStgStride;
            }
            const int col = min(cl, tc::kC - 1) * 12;
            const bool act = cl < nc && (q >= 0);
            float val[3][12];
#pragma unroll
            for (int v = 0; v < 12; v++) {
              val[0][v] = r0[col + v];
              val[1][v] = r1[col + v];
              val[2][v] = r2[col + v];
            }
            const double2 pr = pt.p[(c0 + min(cl, nc - 1)) / ga.nsrc];
            float fl = 0.f, fm = 0.f, fr = 0.f;
            point_forms(pg, (float)(pr.x * pr.x), (float)pr.y, val, fl, fm, fr);
            if (act) {
              tl += fl;
              tm += fm;
              tr += fr;
            }
          }
        }
        racc[0] += (double)tl;
        racc[1] += (double)tm;
        racc[2] += (double)tr;
      }
      // ---- g_{m, anchor a} += sum_q SF_a(q) W_q racc_m(q)
      double v[12];
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int m = 0; m < 3; m++) v[3 * a + m] = pg.wsf[a] * racc[m];
#pragma unroll
      for (int k = 0; k < 12; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[k] = x;
      }
      if (lane == 0)
        for (int k = 0; k < 12; k++) red[k][warp] = v[k];
      named_bar(1, tc::kEpiThreads);
      if (tid < 12) {
        double x = 0.0;
        for (int w = 0; w < 12; w++) x += red[tid][w];
        const int a = tid / 3, m = tid % 3;
        const int anchor = (a == 0 ? ie.x : a == 1 ? ie.y : a == 2 ? ie.z : ie.w) - 1;
        atomicAdd(&grad[(size_t)m * ga.nnpg + anchor], x);
      }
      named_bar(1, tc::kEpiThreads);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == tc::kMmaWarp) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kTmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// host: A tables (SHL in tf32 hi/lo, K-major canonical layout, 4 chains)
// ---------------------------------------------------------------------------
static uint32_t host_tf32(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if ((b & 0x7f800000u) == 0x7f800000u) return b & 0xffffe000u;
  b += 0x1000u;  // round half away from zero on the 13 dropped bits
  return b & 0xffffe000u;
}

std::vector<uint8_t> build_tc_tables(const Tables &t) {
  std::vector<uint8_t> buf(tc::kTabBytes, 0);
  // A' = [A_hi | A_lo], segments of 28 columns (nodes 25-27 zero)
  auto put = [&](int chain, int row, int a, double x) {
    const float xf = (float)x;
    const uint32_t hi = host_tf32(xf);
    float hif;
    std::memcpy(&hif, &hi, 4);
    const uint32_t lo = host_tf32(xf - hif);
    const uint32_t part[2] = {hi, lo};
    for (int g = 0; g < 2; g++) {
      const size_t off = (size_t)chain * tc::kAChain + kmajor_off(row, a + tc::kSeg * g, tc::kALbo);
      std::memcpy(&buf[off], &part[g], 4);
    }
  };
  for (int d = 0; d < 3; d++) {
    const int comp = d == 0 ? 2 : d - 1;  // SHL(3,...) = N, SHL(1,...) = dN/dxi, SHL(2,...) = dN/deta
    for (int q = 0; q < kNq; q++) {
      for (int a = 0; a < kNen; a++) {
        const double x = t.shl[3 * ((size_t)a + (size_t)kNen * q) + comp];
        if (q < 128)
          put(d, q, a, x);
        else
          put(3, tail_lane(d, q - 128), a, x);
      }
      // column 25 carries the centre node's value: weight 1 in the value
      // rows (the shape functions sum to 1), 0 in the derivative rows
      if (d == 0) {
        if (q < 128)
          put(d, q, tc::kRefCol, 1.0);
        else
          put(3, tail_lane(d, q - 128), tc::kRefCol, 1.0);
      }
    }
  }
  // producer slot -> item map.  Item (combo c, field f, node a) = c*50 + f*25
  // + a writes rows c*12 + f*6 + (0..5) at columns a, a+28, a+56; the bank of
  // a store is 4 * (row mod 8) + (column mod 4), so items are grouped by
  // (row0 mod 8, a mod 4) and each 32-slot group (one warp, one j) takes the
  // least-used class with the most items left.
  std::vector<std::vector<int>> cls(16);
  for (int it = 0; it < tc::kC * 2 * kNen; it++) {
    const int cf = it / kNen, a = it % kNen;
    cls[(((6 * cf) & 7) / 2) * 4 + (a & 3)].push_back(it);
  }
  std::vector<int> slot(tc::kItemSlots, -1);
  for (int j = 0; j < tc::kNodeItems; j++)
    for (int w = 0; w < tc::kProdThreads / 32; w++) {
      int used[16] = {0};
      for (int l = 0; l < 32; l++) {
        int best = -1;
        for (int c = 0; c < 16; c++) {
          if (cls[c].empty()) continue;
          if (best < 0 || used[c] < used[best] ||
              (used[c] == used[best] && cls[c].size() > cls[best].size()))
            best = c;
        }
        if (best < 0) break;
        used[best]++;
        slot[w * 32 + l + j * tc::kProdThreads] = cls[best].back();
        cls[best].pop_back();
      }
    }
  std::memcpy(&buf[tc::kABytes], slot.data(), sizeof(int) * tc::kItemSlots);
  return buf;
}

// One-time set-up of the split-precision gradient: checks the DOF layout and
// uploads the SHL tables (a synchronous copy, so it runs outside any stream
// capture).  cudaErrorNotSupported when the layout does not allow the run
// gather.
cudaError_t prepare_grad_tc(Ctx *c) {
  if (c->d_tc_tab) return cudaSuccess;
  // the gather reads a node's three DOFs as one run: LM(3a+1..3a+3) must be
  // d, d+1, d+2 or 0, 0, 0 (what GENID produces)
  for (size_t i = 0; i + 2 < c->h_lm.size(); i += 3) {
    const int d = c->h_lm[i];
    const bool ok = d > 0 ? (c->h_lm[i + 1] == d + 1 && c->h_lm[i + 2] == d + 2)
                          : (c->h_lm[i + 1] == 0 && c->h_lm[i + 2] == 0);
    if (!ok) return cudaErrorNotSupported;
  }
  cudaError_t e;
  std::vector<uint8_t> h = build_tc_tables(c->tab);
  if ((e = cudaFuncSetAttribute(k_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc::kSmemBytes)))
    return e;
  uint8_t *d = nullptr;
  if ((e = cudaMalloc(&d, h.size()))) return e;
  if ((e = cudaMemcpy(d, h.data(), h.size(), cudaMemcpyHostToDevice))) {
    cudaFree(d);
    return e;
  }
  c->d_tc_tab = d;
  return cudaSuccess;
}

cudaError_t launch_grad_tc(Ctx *c, const PairTable &pt, int npairs, int nsrc, const double *u,
                           const double *lam, double *grad, cudaStream_t st) {
  if (!c->d_tc_tab) return cudaErrorNotReady;
  if (c->n_nonpml == 0) return cudaSuccess;
  if ((long long)npairs * nsrc > (1LL << 30)) return cudaErrorInvalidValue;
  TcArgs ga;
  ga.npairs = npairs;
  ga.nsrc = nsrc;
  ga.ndof = c->ndof;
  ga.nnpg = c->nnpg;
  ga.n_elem = c->n_nonpml;
  ga.ncombo = npairs * nsrc;
  ga.inject = c->wait_inject;
  ga.spin = c->wait_limit > 0 ? c->wait_limit : kTcSpinCycles;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int grid = std::min(nsm, c->n_nonpml);
  k_grad_tc<<<grid, tc::kThreads, tc::kSmemBytes, st>>>(c->mv, c->dt, ga, c->d_nonpml, c->d_lm,
                                                         pt, (const double2 *)u,
                                                         (const double2 *)lam, c->d_tc_tab, grad,
                                                         c->d_err);
  return cudaGetLastError();
}

}  // namespace fem25
