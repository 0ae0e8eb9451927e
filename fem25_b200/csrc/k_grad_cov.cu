// Exact lambda/mu/rho adjoint gradient through per-element field
// covariances: a tcgen05 accumulation in split precision (3xTF32, FP32 in
// TMEM, FP64 across (omega, py) pairs) followed by an FP64 contraction.
//
// For an element outside the PML the 2.5D operator is affine in the pair
// weights (estiff25.f:64-154): A = K0 + i wpy K1 - w^2 M + wpy^2 Mc with
// w = omega, wpy = omega * py, and every part is bilinear in the nodal
// values.  The gradient sum over pairs p and sources s,
//     g_m = sum_{p,s} Re( lam_ps^H (dA_p/dm) u_ps ),
// therefore only needs, per element, the weighted covariances of the nodal
// fields (c, d: component of lam, u; i, j: element node; C = conj(lam) u^T)
//     R_cd = sum Re C_cd              (c,d) in {00, 02, 20, 22, 11}
//     P_c  = sum wpy^2 Re C_cc        W_c = sum w^2 Re C_cc
//     I_cd = sum wpy Im C_cd          (c,d) in {01, 21, 10, 12}
// fifteen 25 x 25 blocks whose sums run over every (pair, source) of every
// call, and one contraction of the blocks with the shape-function tables,
// the inverse Jacobian and the anchor weights W_q SF_a(q) at the 169
// points (the bilinear forms of KM25ISOQ, estiff25.f:64-154, written out in
// the blocks).  The per-(element, pair, source) work is a rank-2 real update
// -- a GEMM over the sources -- instead of interpolating both fields at the
// 169 points.
//
// Accumulation (k_grad_cov): one persistent CTA per SM.  Per element and
// pair, D[lam row][u column] += sum_k A[row][k] B[column][k] with
// K = (source, two real parts).  Only nine (lam component, u component,
// Re / Im) products are needed, and they fit one 75 x 75 product when the
// u components enter as
//     B[a][2s, 2s+1]      = (Re u0, Im u0)     slot 0
//     B[32 + a][..]       = (Im u1, -Re u1)    slot 1
//     B[64 + a][..]       = (Re u2, Im u2)     slot 2
// and the lam components as (Re, Im) for components 0 and 2 and as
// (-Im lam1, Re lam1) for component 1 (rows 32 c + a; component 1 again at
// rows 96 + a): row c = 0 then gives Re C00, Im C01, Re C02 in slots 0-2,
// c = 2 gives Re C20, Im C21, Re C22, and c = 1 gives Im C10, -Re C11,
// Im C12.  M = 128, N = 96, 8 sources (K = 16) per stage, x = hi + lo with
// D = A_hi B_hi + A_lo B_hi + A_hi B_lo.
//   loader (warp 7, one thread)  fetches each stage's nodal values with
//                TMA loads -- per element a precomputed list of boxes, 8
//                source rows each, from u and from lam -- into a raw ring of
//                kRawD stages.  GENID numbers an interior element's nodes as
//                one run of 20 consecutive nodes (its own) and five nodes
//                four apart (the column shared with the previous element),
//                so such an element takes two boxes per field: a 20-node 2D
//                box and a 5-node 3D box with a 4-node stride; other
//                elements take boxes of 16-, 4- and 1-node runs.
//   MMA (warp 3, one thread)  issues the MMAs into one of 4 TMEM
//                accumulators of 128 columns (each takes kDrain stages of
//                one pair)
//   7 converter warps  thread (node, source) reads its node's six complex
//                values from the raw stage and writes them (FP64 -> tf32
//                hi/lo, signs and swaps above) into one of 3 operand stages
//   15 epilogue warps  one block each: the warp's TMEM lane quarter holds
//                the lam component (lane = node); it reads its 25 columns
//                and adds them, weighted (and signed) by the pair, into 25
//                FP64 registers; at the end of the element it writes (or
//                adds) the block row to memory.
// Measured per stage (clock stamps per role): a TMA box costs the issuing
// thread about 150 cycles whatever its size, so seven boxes per field (16-,
// 4- and five 1-node runs) took longer than the stage's conversion, and
// issuing them from the MMA thread serialised loads and MMAs; 16-byte
// cp.async gathers from one warp were slower still (about 100 cycles per
// warp instruction).  Hence the loader warp and the two-box plan.
// Hand-offs are mbarriers (the raw stages complete by TMA transaction
// bytes); every wait is bounded and a wait that runs out sets the error
// word and drains the schedule without waiting (the loader stops issuing
// and waits, bounded, for the loads in flight before the CTA exits).
//
// Contraction (k_grad_cov_fin, FP64): per element the blocks are combined
// (symmetric parts of R_00, R_22, R_11; S = R_02 + R_20^T;
// G_1 = I_01 - I_10^T, G_2 = I_21 - I_12^T; P_1, P_0 + P_2, W_0 + W_1 + W_2)
// and each is contracted with the tensor-product shape functions,
// N_a(xi_x, eta_z) = l_ax(xi_x) l_ae(eta_z) (dshl.f:100-243), by sum
// factorisation: Z = B l_e, Y = Z l_x, F(q) = T(q)^T Y(q), about 0.6 M FMA
// per element, independent of the number of pairs and sources.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "kcommon.cuh"
#include "tcgen05.cuh"

namespace fem25 {

namespace cov {
constexpr int kG = 8;                        // sources per stage
constexpr int kK = 2 * kG;                   // K columns per stage
constexpr int kM = 128;
constexpr int kN = 96;                       // B rows: slot k (u component k) at rows 32 k + node
constexpr uint32_t kALbo = kM / 8 * 128;     // 2048 B between K chunks of A
constexpr uint32_t kBLbo = kN / 8 * 128;     // 1536 B between K chunks of B
constexpr int kATile = (int)kALbo * (kK / 4);  // 8 KB
constexpr int kBTile = (int)kBLbo * (kK / 4);  // 6 KB
constexpr int kStage = 2 * kATile + 2 * kBTile;  // A_hi, A_lo, B_hi, B_lo: 28 KB
constexpr int kNB = 3;                       // operand stages in the ring
constexpr int kNodeBytes = 48;               // one node's three complex128 DOFs
constexpr int kRawField = kNen * kG * kNodeBytes;  // 9600 B: 25 nodes x 8 sources
constexpr int kRawStage = 2 * kRawField;     // u then lam
constexpr int kRawD = 5;                     // raw stages in the ring
constexpr int kSmemBytes = kNB * kStage + kRawD * kRawStage;  // 180 KB
constexpr int kThreads = 768;                // 24 warps
constexpr int kMmaWarp = 3;
constexpr int kLoadWarp = 7;
constexpr int kEpiWarps = 15;
constexpr int kProdWarps = 7;
constexpr int kDrain = 2;                    // stages per TMEM accumulation (FP32 sums of 2 kDrain kG)
constexpr int kUnits = 4;                    // TMEM accumulators
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kTmemUnit = 128;          // columns per accumulator (96 used)
constexpr int kBlocks = 15;
constexpr int kBlk = kNen * kNen + 1;        // 625 doubles per block, padded to 16 bytes
// gather boxes by code: 2D runs of 16, 4, 1 and 20 nodes; 3D: 5 nodes with
// a stride of 4 nodes (kStrideNodes)
constexpr int kNCodes = 5;
constexpr int kBoxNodes[kNCodes] = {16, 4, 1, 20, 5};
constexpr int kStrideNodes = 4;
constexpr int kRefNode = 12;                 // the element's centre node: the reference values
static_assert(kProdWarps * 32 >= (kNen + 1) * kG, "one converter thread per (node row, source)");
static_assert(kRawField % 128 == 0, "raw regions start on 128-byte boundaries");
static_assert(kSmemBytes <= 227 * 1024, "shared memory");
static_assert(kUnits * kTmemUnit <= kTmemCols, "tensor memory");
}  // namespace cov

constexpr uint32_t kCovIdesc = tf32_idesc(cov::kM, cov::kN);

// Epilogue block k (0-4) of lam component c: the block it accumulates
// (index into R00 R02 R20 R22 R11 P0 P1 P2 W0 W1 W2 I01 I21 I10 I12), its
// u slot (TMEM column 32 slot), its weight (0: 1, 1: wpy^2, 2: w^2, 3: wpy)
// and whether the product enters with a minus sign (component 1's slot 1
// holds -Re C11).
__device__ __forceinline__ void cov_role(int c, int k, int &blk, int &slot, int &wt, bool &neg) {
  neg = false;
  switch (c * 5 + k) {
    case 0: blk = 0; slot = 0; wt = 0; break;               // lam_0: R00
    case 1: blk = 1; slot = 2; wt = 0; break;               //        R02
    case 2: blk = 5; slot = 0; wt = 1; break;               //        P0
    case 3: blk = 8; slot = 0; wt = 2; break;               //        W0
    case 4: blk = 11; slot = 1; wt = 3; break;              //        I01
    case 5: blk = 4; slot = 1; wt = 0; neg = true; break;   // lam_1: R11
    case 6: blk = 13; slot = 0; wt = 3; break;              //        I10
    case 7: blk = 6; slot = 1; wt = 1; neg = true; break;   //        P1
    case 8: blk = 9; slot = 1; wt = 2; neg = true; break;   //        W1
    case 9: blk = 14; slot = 2; wt = 3; break;              //        I12
    case 10: blk = 2; slot = 0; wt = 0; break;              // lam_2: R20
    case 11: blk = 3; slot = 2; wt = 0; break;              //        R22
    case 12: blk = 7; slot = 2; wt = 1; break;              //        P2
    case 13: blk = 10; slot = 2; wt = 2; break;             //        W2
    default: blk = 12; slot = 1; wt = 3; break;             //        I21
  }
}

// Warp roles.  A warp reads the TMEM lanes of its quarter (warp % 4), which
// is also its scheduler partition.  The lam rows of component c sit in lane
// quarter c, and those of component 1 a second time in quarter 3, so the 15
// epilogue warps take partitions 0 (component 0, five blocks), 1 (component
// 1, three blocks), 2 (component 2, five blocks) and 3 (component 1, two
// blocks); the MMA and loader warps sit on partition 3 and the 7 converter
// warps spread 1 / 3 / 1 / 2 over the partitions.  24 warps at 80 registers
// fill a partition's 16 K registers (a 25th warp would not fit).
// Returns 0 (epilogue: component c, block k of it), 1 (MMA), 2 (converter
// number pidx) or 3 (loader).
__device__ __forceinline__ int cov_warp_role(int w, int &c, int &k, int &pidx) {
  const int q = w & 3, r = w >> 2;  // partition, rank on it (0..5)
  c = k = pidx = 0;
  if (q == 0 || q == 2) {
    if (r < 5) {
      c = q;
      k = r;
      return 0;
    }
    pidx = q == 0 ? 0 : 1;  // warps 20, 22
    return 2;
  }
  if (q == 1) {
    if (r < 3) {
      c = 1;
      k = r;  // blocks 0-2 of component 1
      return 0;
    }
    pidx = 2 + (r - 3);  // warps 13, 17, 21
    return 2;
  }
  if (r == 0) return 1;  // warp 3
  if (r == 1) return 3;  // warp 7
  if (r < 4) {
    c = 1;
    k = r + 1;  // blocks 3, 4 of component 1, lane quarter 3 (warps 11, 15)
    return 0;
  }
  pidx = 5 + (r - 4);  // warps 19, 23
  return 2;
}

// Scaling.  FP32 sums of products of small fields underflow: solved fields
// in SI units (displacements per newton ~1e-10, adjoint fields ~1e-20) give
// products near FP32's smallest normal numbers, where the split's low parts
// are flushed.  Each pair's u and lam therefore enter the tensor cores scaled
// by powers of two that bring their largest sampled component to [1, 2)
// (exact in FP64), and the epilogue multiplies the pair's weight back.
constexpr int kExpBias = 4096;    // exponents stored with this offset (0: all zero)
// every 251st complex value of a field is sampled: the scale only has to
// put the fields' magnitudes well inside FP32's range, and sampling more
// densely cost a measurable part of the accumulation (0.45 ms at 1 in 13
// for 2 x 32 fields of 2.3 M DOF)
constexpr int kScaleStride = 251;

__device__ __forceinline__ double cov_scale_of(int e) {
  return e == 0 ? 1.0 : ldexp(1.0, kExpBias - e);
}

struct CovArgs {
  const int *exps;  // [pair][u, lam]: sampled binary exponents (+ kExpBias)
  int npairs, nsrc, ndof, n_elem;
  int add;          // 1: add into the accumulators, 0: overwrite them
  int inject;       // 1: converter warp 0 of CTA 0 withholds its first stage
                    // arrival, so the MMA thread's wait runs out (a test of
                    // the time-out path)
  long long spin;   // SM clocks a pipeline wait may take before it gives up
};

// The TMA views of the launch's fields: [field: u, lam][box code].  Codes
// 0-3: 2D, a row of 2 NDOF doubles per (pair, source), box = (6 x width
// doubles, kG rows); code 4: 3D, (24 doubles = 4 nodes, NDOF / 4 node
// groups of 192 bytes, rows), box = (6, 5, kG).
struct CovMaps {
  CUtensorMap m[2][cov::kNCodes];
};

// Per-element gather plan (elements outside the PML, kernel order):
//   op = {x: first double of the box (2 (DOF - 1)), code | raw 128-B granule << 8}
//   node[a] = raw byte offset of the node's source-0 values | box code << 16,
//             or 0xFFFFFFFF for a node without DOFs (fixed)
//   tx = TMA bytes of one stage (both fields)
struct CovPlan {
  const int2 *ops;
  const int *opptr;    // [n_elem + 1]
  const uint32_t *node;  // [n_elem][25]
  const int *tx;       // [n_elem]
};

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(mbar),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            int z, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(mbar)
      : "memory");
}

// the tf32 part of x, rounded to nearest (ties away from zero) on the bit
// pattern; finite inputs only
__device__ __forceinline__ uint32_t tf32_hi(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}

// bytes of one source row of a box
__device__ __forceinline__ uint32_t cov_box_row_bytes(uint32_t code) {
  return code == 0 ? 768u : code == 1 ? 192u : code == 2 ? 48u : code == 3 ? 960u : 240u;
}

__global__ void __launch_bounds__(cov::kThreads, 1)
    k_grad_cov(const __grid_constant__ CovMaps maps, CovArgs ga, CovPlan plan, PairTable pt,
               double *__restrict__ acc_out, int *__restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm_dyn[];
  // 128-byte aligned base (TMA destinations); the launch adds 128 bytes
  uint8_t *sm = sm_dyn + ((128u - (smem_u32(sm_dyn) & 127u)) & 127u);
  __shared__ uint64_t bar_bfull[cov::kNB], bar_bempty[cov::kNB];
  __shared__ uint64_t bar_rfull[cov::kRawD], bar_rempty[cov::kRawD];
  __shared__ uint64_t bar_tfull[cov::kUnits], bar_tempty[cov::kUnits];
  __shared__ uint64_t bar_drain;
  __shared__ uint32_t tmem_base_s;
  __shared__ int drain_s;
  __shared__ double2 scale_s[kMaxPairs];  // per pair: (u, lam) scales
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  volatile int *drain = &drain_s;
  for (int p = tid; p < ga.npairs; p += blockDim.x)
    scale_s[p] = make_double2(cov_scale_of(ga.exps[2 * p]), cov_scale_of(ga.exps[2 * p + 1]));

  // ---- set-up: zeroed stages (rows and columns no conversion writes stay
  // zero), barriers, TMEM
  for (int i = tid * 16; i < cov::kSmemBytes; i += cov::kThreads * 16)
    *reinterpret_cast<uint4 *>(sm + i) = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    drain_s = 0;
    // multi-warp hand-offs count warps: each warp syncs, then one lane arrives
    for (int b = 0; b < cov::kNB; b++) {
      mbar_init(smem_u32(&bar_bfull[b]), cov::kProdWarps);
      mbar_init(smem_u32(&bar_bempty[b]), 1);
    }
    for (int b = 0; b < cov::kRawD; b++) {
      mbar_init(smem_u32(&bar_rfull[b]), 1);
      mbar_init(smem_u32(&bar_rempty[b]), cov::kProdWarps);
    }
    for (int b = 0; b < cov::kUnits; b++) {
      mbar_init(smem_u32(&bar_tfull[b]), 1);
      mbar_init(smem_u32(&bar_tempty[b]), cov::kEpiWarps);
    }
    mbar_init(smem_u32(&bar_drain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == cov::kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(cov::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const int nch = (ga.nsrc + cov::kG - 1) / cov::kG;  // stages per (element, pair)
  const int my_elems = (ga.n_elem - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const uint32_t total = (uint32_t)max(my_elems, 0) * (uint32_t)ga.npairs * (uint32_t)nch;
  uint8_t *raw = sm + cov::kNB * cov::kStage;
  int rc, rk, rp;
  const int role = cov_warp_role(warp, rc, rk, rp);

  if (role == 2) {
    // =================== converters (warps 13, 17, 19, 20-23)
    // A thread owns node row a and source g of every stage (row 25: the
    // reference values; a = 26: idle): it reads the node's u and lam values
    // of source g from the raw stage (the node's box and place in it come
    // from the element's plan) and writes them (FP64 -> tf32 hi/lo) into A
    // rows 32c + a (lam; component 1 also at 96 + a) and B rows 32c + a (u)
    // at K = 2g.  Converters 0-3 take rows 0-15 (lanes: a mod 8, g mod 2,
    // a / 8), 4-5 rows 16-23 (a mod 8, g mod 4) and 6 rows 24-25 with half
    // its lanes, so a warp's threads cover the 16 (row mod 8, g mod 2)
    // shared-memory bank classes evenly and each 8-byte tile store is two
    // wavefronts (four for converter 6).
    int a, g;
    if (rp < 4) {
      a = ((lane >> 4) & 1) * 8 + (lane & 7);
      g = 2 * rp + ((lane >> 3) & 1);
    } else if (rp < 6) {
      a = 16 + (lane & 7);
      g = 4 * (rp - 4) + (lane >> 3);
    } else {
      a = lane < 16 ? 24 + (lane & 1) : kNen + 1;
      g = (lane >> 1) & 7;
    }
    const bool node = a < kNen;    // a node's deviation from the reference node
    const bool refw = a == kNen;   // the reference values themselves (row / slot row 25)
    const uint32_t to_a = kmajor_off(a, 2 * g, cov::kALbo);                        // A row a
    const uint32_t to_b = 2 * cov::kATile + kmajor_off(a, 2 * g, cov::kBLbo);      // B row a
    auto node_info = [&](int e, int n) -> uint32_t {
      return e < ga.n_elem ? __ldg(plan.node + (size_t)e * kNen + n) : 0xFFFFFFFFu;
    };
    int iei = blockIdx.x, ip = 0, ich = 0;
    // plan entries of this thread's node and of the reference node, for the
    // current element and (prefetched) the next one
    uint32_t ni = node ? node_info(iei, a) : 0xFFFFFFFFu;
    uint32_t nr = node_info(iei, cov::kRefNode);
    uint32_t ni_next = node ? node_info(iei + gridDim.x, a) : 0xFFFFFFFFu;
    uint32_t nr_next = node_info(iei + gridDim.x, cov::kRefNode);
    auto raw_of = [&](uint32_t info, int rs) -> const uint8_t * {
      return raw + rs * cov::kRawStage + (info & 0xFFFFu) + g * cov_box_row_bytes(info >> 16);
    };
    for (uint32_t s = 0; s < total; s++) {
      const int rs = (int)(s % cov::kRawD), bs = (int)(s % cov::kNB);
      mbar_wait(smem_u32(&bar_rfull[rs]), (s / cov::kRawD) & 1u, drain, err, -2000006, ga.spin);
      // every raw value of the stage first (the loads in flight together),
      // then the raw slot is released and the operand stage awaited
      const bool gact = g < ga.nsrc - ich * cov::kG;
      const bool vact = gact && node && ni != 0xFFFFFFFFu;
      const double2 scl = scale_s[ip];
      const double su = scl.x, sl = scl.y;
      const bool ract = gact && (node || refw) && nr != 0xFFFFFFFFu;
      float xv[6][2];
      {
        const uint8_t *src = vact ? raw_of(ni, rs) : raw;
        const uint8_t *rsrc = ract ? raw_of(nr, rs) : raw;
        double2 rv[6], vv[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {  // j < 3: u component j; else lam component j - 3
          const int fo = (j < 3 ? 0 : cov::kRawField) + 16 * (j % 3);
          rv[j] = ract ? *reinterpret_cast<const double2 *>(rsrc + fo) : make_double2(0.0, 0.0);
          vv[j] = vact ? *reinterpret_cast<const double2 *>(src + fo) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int j = 0; j < 6; j++) {
          // node threads store the deviation (a fixed node's value is 0),
          // reference writers the reference values
          const double sc = j < 3 ? su : sl;
          const double2 v = node ? make_double2((vv[j].x - rv[j].x) * sc, (vv[j].y - rv[j].y) * sc)
                                 : make_double2(rv[j].x * sc, rv[j].y * sc);
          float x0 = (float)v.x, x1 = (float)v.y;
          // the sign / swap of the layout: u1 -> (Im, -Re), lam1 -> (-Im, Re)
          if (j % 3 == 1) {
            const float t = x0;
            x0 = j < 3 ? x1 : -x1;
            x1 = j < 3 ? -t : t;
          }
          xv[j][0] = x0;
          xv[j][1] = x1;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bar_rempty[rs]));
      mbar_wait(smem_u32(&bar_bempty[bs]), ((s / cov::kNB) & 1u) ^ 1u, drain, err, -2000001,
                ga.spin);
      if (node || refw) {
        uint8_t *st = sm + bs * cov::kStage;
#pragma unroll
        for (int j = 0; j < 6; j++) {
          const int c = j % 3;
          // x = hi + lo: hi = x rounded to 10 mantissa bits (integer
          // round-half-up on the bit pattern), lo = x - hi exactly; the MMA
          // reads lo's top 19 bits
          const float x0 = xv[j][0], x1 = xv[j][1];
          const uint32_t h0 = tf32_hi(x0), h1 = tf32_hi(x1);
          const uint32_t l0 = __float_as_uint(x0 - __uint_as_float(h0));
          const uint32_t l1 = __float_as_uint(x1 - __uint_as_float(h1));
          if (j < 3) {  // u -> B row 32c + a, hi then lo
            uint8_t *d = st + to_b + 512 * c;
            *reinterpret_cast<uint2 *>(d) = make_uint2(h0, h1);
            *reinterpret_cast<uint2 *>(d + cov::kBTile) = make_uint2(l0, l1);
          } else {  // lam -> A row 32c + a (hi, then lo); component 1 also to row 96 + a
            uint8_t *d = st + to_a + 512 * c;
            *reinterpret_cast<uint2 *>(d) = make_uint2(h0, h1);
            *reinterpret_cast<uint2 *>(d + cov::kATile) = make_uint2(l0, l1);
            if (c == 1) {
              *reinterpret_cast<uint2 *>(d + 1024) = make_uint2(h0, h1);
              *reinterpret_cast<uint2 *>(d + 1024 + cov::kATile) = make_uint2(l0, l1);
            }
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      const bool withhold = ga.inject && blockIdx.x == 0 && rp == 0 && s == 0;
      if (lane == 0 && !withhold) mbar_arrive(smem_u32(&bar_bfull[bs]));
      if (++ich == nch) {
        ich = 0;
        if (++ip == ga.npairs) {
          ip = 0;
          iei += gridDim.x;
          ni = ni_next;
          nr = nr_next;
          ni_next = node ? node_info(iei + gridDim.x, a) : 0xFFFFFFFFu;
          nr_next = node_info(iei + gridDim.x, cov::kRefNode);
        }
      }
    }
  } else if (role == 3) {
    // =================== loader (lane 0 issues the TMA loads; lane k holds
    // box k of the element, prefetched an element ahead)
    const uint32_t rbase = smem_u32(raw);
    if (lane == 0)
      for (int f = 0; f < 2; f++)
        for (int cd = 0; cd < cov::kNCodes; cd++)
          asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.m[f][cd]))
                       : "memory");
    auto load_ops = [&](int e, int2 &op, int &n, uint32_t &tx) {
      op = make_int2(0, 0);
      n = 0;
      tx = 0;
      if (e < ga.n_elem) {
        const int k0 = __ldg(plan.opptr + e);
        n = __ldg(plan.opptr + e + 1) - k0;
        if (lane < n) op = __ldg(plan.ops + k0 + lane);
        tx = (uint32_t)__ldg(plan.tx + e);
      }
    };
    int iei = blockIdx.x, ip = 0, ich = 0;
    int2 op_cur, op_nxt;
    int n_cur, n_nxt;
    uint32_t tx_cur, tx_nxt;
    load_ops(iei, op_cur, n_cur, tx_cur);
    load_ops(iei + (int)gridDim.x, op_nxt, n_nxt, tx_nxt);
    uint32_t issued = 0;
    for (; issued < total; issued++) {
      const int rs = (int)(issued % cov::kRawD);
      if (issued >= (uint32_t)cov::kRawD)
        mbar_wait(smem_u32(&bar_rempty[rs]), ((issued / cov::kRawD) & 1u) ^ 1u, drain, err,
                  -2000007, ga.spin);
      if (__shfl_sync(0xffffffffu, *drain, 0)) break;  // no new loads once the CTA drains
      const uint32_t full = smem_u32(&bar_rfull[rs]);
      if (lane == 0) mbar_arrive_expect_tx(full, tx_cur);
      const int y = ip * ga.nsrc + ich * cov::kG;
      const uint32_t dst0 = rbase + (uint32_t)(rs * cov::kRawStage);
      for (int k = 0; k < n_cur; k++) {
        const int x = __shfl_sync(0xffffffffu, op_cur.x, k);
        const int yk = __shfl_sync(0xffffffffu, op_cur.y, k);
        if (lane == 0) {
          const int code = yk & 0xFF;
          const uint32_t d = dst0 + (uint32_t)(yk >> 8) * 128u;
          if (code == 4) {  // x = 6 n for the first node n: group n / 4, double 6 (n % 4)
            tma_load_3d(d, &maps.m[0][4], x % 24, x / 24, y, full);
            tma_load_3d(d + cov::kRawField, &maps.m[1][4], x % 24, x / 24, y, full);
          } else {
            tma_load_2d(d, &maps.m[0][code], x, y, full);
            tma_load_2d(d + cov::kRawField, &maps.m[1][code], x, y, full);
          }
        }
      }
      __syncwarp();
      if (++ich == nch) {
        ich = 0;
        if (++ip == ga.npairs) {
          ip = 0;
          iei += gridDim.x;
          op_cur = op_nxt;
          n_cur = n_nxt;
          tx_cur = tx_nxt;
          load_ops(iei + (int)gridDim.x, op_nxt, n_nxt, tx_nxt);
        }
      }
    }
    // loads still in flight (a drained CTA may have issued stages nobody
    // consumed): wait, bounded, for the last phase issued into each raw slot
    if (lane == 0 && *drain) {
      for (int r = 0; r < cov::kRawD; r++) {
        const uint32_t n = issued > (uint32_t)r ? (issued - 1 - (uint32_t)r) / cov::kRawD + 1 : 0u;
        if (n == 0) continue;
        const long long t0 = clock64();
        while (!mbar_try_wait(smem_u32(&bar_rfull[r]), (n - 1) & 1u)) {
          if (clock64() - t0 > kTcSpinCycles) {
            atomicCAS(err, 0, -2000008);
            break;
          }
        }
      }
    }
    __syncwarp();
  } else if (role == 1) {
    // =================== MMA issuer (lane 0 issues the MMAs and commits)
    const uint32_t sbase = smem_u32(sm);
    const uint64_t adesc = umma_desc(sbase, cov::kALbo, 128);
    const uint64_t bdesc = umma_desc(sbase, cov::kBLbo, 128);
    uint32_t s = 0, unit = 0;
    for (int ei = blockIdx.x; ei < ga.n_elem; ei += gridDim.x) {
      for (int p = 0; p < ga.npairs; p++) {
        for (int ch = 0; ch < nch; ch++, s++) {
          // a TMEM accumulator takes kDrain stages of one pair (FP32 sums
          // of at most 2 kDrain kG products), then the epilogue adds it in FP64
          const bool first = ch % cov::kDrain == 0;
          const bool last = ch % cov::kDrain == cov::kDrain - 1 || ch == nch - 1;
          const int ts = (int)(unit % cov::kUnits), bs = (int)(s % cov::kNB);
          if (first)
            mbar_wait(smem_u32(&bar_tempty[ts]), ((unit / cov::kUnits) & 1u) ^ 1u, drain, err,
                      -2000002, ga.spin);
          mbar_wait(smem_u32(&bar_bfull[bs]), (s / cov::kNB) & 1u, drain, err, -2000003, ga.spin);
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          if (lane == 0) {
            const uint32_t td = tmem + (uint32_t)ts * cov::kTmemUnit;
            const int nact = min(cov::kG, ga.nsrc - ch * cov::kG);
            const int nks = (nact + 3) / 4;  // K steps of 8 = 4 sources
            const uint32_t so = (uint32_t)(bs * cov::kStage);
            for (int ks = 0; ks < nks; ks++) {
              const uint64_t ahi = adesc + (uint64_t)((so + 2 * ks * cov::kALbo) >> 4);
              const uint64_t alo = ahi + (uint64_t)(cov::kATile >> 4);
              const uint64_t bhi =
                  bdesc + (uint64_t)((so + 2 * cov::kATile + 2 * ks * cov::kBLbo) >> 4);
              const uint64_t blo = bhi + (uint64_t)(cov::kBTile >> 4);
              mma_tf32(td, ahi, bhi, kCovIdesc, (first && ks == 0) ? 0u : 1u);
              mma_tf32(td, alo, bhi, kCovIdesc, 1u);
              mma_tf32(td, ahi, blo, kCovIdesc, 1u);
            }
            mma_commit(smem_u32(&bar_bempty[bs]));
            if (last) mma_commit(smem_u32(&bar_tfull[ts]));
          }
          __syncwarp();
          if (last) unit++;
        }
      }
    }
    if (lane == 0) {
      // every MMA issued above has completed once this commit arrives
      mma_commit(smem_u32(&bar_drain));
      const long long t0 = clock64();
      while (!mbar_try_wait(smem_u32(&bar_drain), 0u)) {
        if (clock64() - t0 > kTcSpinCycles) {
          atomicCAS(err, 0, -2000004);
          break;
        }
      }
    }
    __syncwarp();
  } else {
    // =================== epilogue (15 warps)
    int blk, slot, wt;
    bool neg;
    cov_role(rc, rk, blk, slot, wt, neg);
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;  // lane quarter = partition
    // lane a < 25: row a of the deviations' covariance (columns 0-24) and its
    // product with the reference (column 25); lane 25: the reference's
    // product with the deviations (columns 0-24) and with itself (column 25)
    constexpr int kAcc = kNen + 1;
    double acc[kAcc];
#pragma unroll
    for (int j = 0; j < kAcc; j++) acc[j] = 0.0;
    uint32_t unit = 0;  // TMEM accumulations so far
    for (int ei = blockIdx.x; ei < ga.n_elem; ei += gridDim.x) {
      for (int p = 0; p < ga.npairs; p++) {
        const double2 pr = pt.p[p];
        double w = wt == 0 ? 1.0 : wt == 1 ? pr.y * pr.y : wt == 2 ? pr.x * pr.x : pr.y;
        if (neg) w = -w;
        // the pair's scaling undone
        w /= scale_s[p].x * scale_s[p].y;
        for (int ch = 0; ch < nch; ch += cov::kDrain, unit++) {
          const int ts = (int)(unit % cov::kUnits);
          mbar_wait(smem_u32(&bar_tfull[ts]), (unit / cov::kUnits) & 1u, drain, err, -2000005,
                    ga.spin);
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t tb = tmem + lane_base + (uint32_t)ts * cov::kTmemUnit + 32u * (uint32_t)slot;
          __syncwarp();
          uint32_t r[16];
          tmem_ld16(tb, r);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; j++) acc[j] += w * (double)__uint_as_float(r[j]);
          tmem_ld16(tb + 16u, r);
          tmem_wait_ld();
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[ts]));
#pragma unroll
          for (int j = 16; j < kAcc; j++) acc[j] += w * (double)__uint_as_float(r[j - 16]);
        }
      }
      // the block of the fields themselves: C_aj = D_aj + D_a,25 + D_25,j + D_25,25
      // (field = reference + deviation), in FP64; lane 25's row comes by shuffle
      const double s_ref = __shfl_sync(0xffffffffu, acc[kNen], kNen);
#pragma unroll
      for (int j = 0; j < kNen; j++) {
        const double bj = __shfl_sync(0xffffffffu, acc[j], kNen);
        acc[j] = acc[j] + acc[kNen] + (bj + s_ref);
      }
      // block row `lane` of this element, stored transposed ([j][i]) so that
      // the 25 lanes of a store are consecutive
      if (lane < kNen) {
        double *dst = acc_out + ((size_t)ei * cov::kBlocks + blk) * cov::kBlk + lane;
        if (ga.add) {
          // this lane is the only writer of these words in the launch (one CTA
          // per element, one warp per block, one lane per row): a plain
          // read-modify-write, the 25 loads in flight together
          double old[kNen];
#pragma unroll
          for (int j = 0; j < kNen; j++) old[j] = dst[kNen * j];
#pragma unroll
          for (int j = 0; j < kNen; j++) dst[kNen * j] = old[j] + acc[j];
        } else {
#pragma unroll
          for (int j = 0; j < kNen; j++) dst[kNen * j] = acc[j];
        }
      }
#pragma unroll
      for (int j = 0; j < kAcc; j++) acc[j] = 0.0;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == cov::kMmaWarp) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cov::kTmemCols)
                 : "memory");
  }
}

// Per pair: the binary exponent (+ kExpBias) of the largest real or
// imaginary part among every kScaleStride-th complex value of u (exps[2p])
// and of lam (exps[2p + 1]) over the pair's sources; 0 if all are zero.
__global__ void k_cov_scale(const double2 *__restrict__ u, const double2 *__restrict__ lam,
                            long long per_pair, int *__restrict__ exps) {
  const int p = blockIdx.y;
  const double2 *up = u + (long long)p * per_pair, *lp = lam + (long long)p * per_pair;
  int eu = 0, el = 0;
  const long long step = (long long)gridDim.x * blockDim.x * kScaleStride;
#pragma unroll 4
  for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * kScaleStride;
       i < per_pair; i += step) {
    const double2 a = up[i], b = lp[i];
    const double ma = fmax(fabs(a.x), fabs(a.y)), mb = fmax(fabs(b.x), fabs(b.y));
    if (ma > 0.0) eu = max(eu, ilogb(ma) + kExpBias);
    if (mb > 0.0) el = max(el, ilogb(mb) + kExpBias);
  }
  for (int o = 16; o > 0; o >>= 1) {
    eu = max(eu, __shfl_xor_sync(0xffffffffu, eu, o));
    el = max(el, __shfl_xor_sync(0xffffffffu, el, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(exps + 2 * p, eu);
    atomicMax(exps + 2 * p + 1, el);
  }
}

// ---------------------------------------------------------------------------
// FP64 contraction of the accumulated blocks
// ---------------------------------------------------------------------------
// Per element and combined block B (9 of them), with the shape functions
// T_t(q)_(ix + 5 ie) = X_t(qx, ix) E_t(qz, ie) for t = N (X = l, E = l),
// xi (l', l), eta (l, l'):
//   Z_A[i][jx][qz]      = sum_je B[i][jx + 5 je] A(qz, je)                A = l, l'
//   W_EA[ix][jx][qz]    = sum_ie E(qz, ie) Z_A[ix + 5 ie][jx][qz]        E = l, l'
//   F^{t1 t2}(qz, qx)   = sum_jx X_t2(qx, jx) sum_ix X_t1(qx, ix) W_{E_t1 A_t2}[ix][jx][qz]
// = T_t1(q)^T B T_t2(q): about 0.28 M FMA per element.
namespace covf {
constexpr int kThreads = 256;
constexpr int kRawMax = 3;                   // raw blocks behind one combined block
constexpr int kRaw = kRawMax * cov::kBlk;    // doubles per raw buffer
constexpr int kZ = kNen * kNl * kNint;       // 1625: Z[i][jx][qz]
constexpr int kW = kNl * kNl * kNint;        // 325: W[ix][jx][qz]
constexpr int kSmemDoubles = 2 * kRaw + 2 * kZ + 4 * kW + 2 * kNint * kNl + 4 * kNq;
constexpr int kSmemBytes = kSmemDoubles * 8;  // 72 KB: three CTAs per SM
}  // namespace covf

// 1D Lagrange factors of the element's shape functions at the 13 points:
// l[q][i] = l_i(x_q), d[q][i] = l_i'(x_q)  (SHL = l(xi) l(eta), dshl.f:100-243)
struct CovFinTabs {
  double l[kNint][kNl];
  double d[kNint][kNl];
};

// raw blocks behind combined block b (stored [j][i]): first index and count
__device__ __forceinline__ void cov_raw_of(int b, int *ids, int &n) {
  switch (b) {
    case 0: ids[0] = 0; n = 1; break;                  // R00
    case 1: ids[0] = 3; n = 1; break;                  // R22
    case 2: ids[0] = 4; n = 1; break;                  // R11
    case 3: ids[0] = 1; ids[1] = 2; n = 2; break;      // R02, R20
    case 4: ids[0] = 11; ids[1] = 13; n = 2; break;    // I01, I10
    case 5: ids[0] = 12; ids[1] = 14; n = 2; break;    // I21, I12
    case 6: ids[0] = 6; n = 1; break;                  // P1
    case 7: ids[0] = 5; ids[1] = 7; n = 2; break;      // P0, P2
    default: ids[0] = 8; ids[1] = 9; ids[2] = 10; n = 3; break;  // W0, W1, W2
  }
}

// combined block b at (i, j) from its raw blocks r (r + k * kBlk: k-th raw)
__device__ __forceinline__ double cov_bval(int b, const double *r, int i, int j) {
  const int ij = j * kNen + i, ji = i * kNen + j;  // r[ij] = R[i][j]
  switch (b) {
    case 0: case 1: case 2: return 0.5 * (r[ij] + r[ji]);           // symmetric part
    case 3: return r[ij] + r[cov::kBlk + ji];                        // R02 + R20^T
    case 4: case 5: return r[ij] - r[cov::kBlk + ji];                // I01 - I10^T, I21 - I12^T
    case 6: return r[ij];
    case 7: return r[ij] + r[cov::kBlk + ij];
    default: return r[ij] + r[cov::kBlk + ij] + r[2 * cov::kBlk + ij];
  }
}

// sum_jx x2[jx] sum_ix x1[ix] W[ix][jx][qz]
__device__ __forceinline__ double cov_fw(const double *W, int qz, const double *x1,
                                         const double *x2) {
  double f = 0.0;
#pragma unroll
  for (int jx = 0; jx < kNl; jx++) {
    double h = 0.0;
#pragma unroll
    for (int ix = 0; ix < kNl; ix++) h = fma(x1[ix], W[(ix * kNl + jx) * kNint + qz], h);
    f = fma(x2[jx], h, f);
  }
  return f;
}

__global__ void __launch_bounds__(covf::kThreads, 3)
    k_grad_cov_fin(MeshView mv, DevTables dt, int n_elem, int nnpg, const int *__restrict__ elems,
                   const double *__restrict__ accb, CovFinTabs tb, double *__restrict__ grad,
                   int *__restrict__ err) {
  extern __shared__ __align__(16) double fs[];
  double *rawb = fs;                          // [2][kRaw]
  double *zl = rawb + 2 * covf::kRaw, *zd = zl + covf::kZ;
  double *wb = zd + covf::kZ;                 // [4][kW]: (E, A) = (l,l) (l,l') (l',l) (l',l')
  double *tl_s = wb + 4 * covf::kW, *td_s = tl_s + kNint * kNl;  // 1D tables
  double *wsf_s = td_s + kNint * kNl;         // [4][169] W_q SF_a(q)
  __shared__ double red[12][covf::kThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int k = tid; k < kNint * kNl; k += covf::kThreads) {
    tl_s[k] = tb.l[k / kNl][k % kNl];
    td_s[k] = tb.d[k / kNl][k % kNl];
  }
  const bool ptq = tid < kNq;
  const int q = ptq ? tid : 0, qx = q % kNint, qz = q / kNint;
  const int my_elems = (n_elem - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int ntask = max(my_elems, 0) * 9;     // tasks (element, combined block)

  // copies the raw blocks of task k into raw buffer k & 1 (16-byte cp.async)
  auto fetch = [&](int k) {
    if (k < ntask) {
      const int ei = (int)blockIdx.x + (k / 9) * (int)gridDim.x, b = k % 9;
      int ids[covf::kRawMax], n;
      cov_raw_of(b, ids, n);
      double *dst = rawb + (k & 1) * covf::kRaw;
      const double *src = accb + (size_t)ei * cov::kBlocks * cov::kBlk;
      constexpr int kV = cov::kBlk / 2;  // 16-byte vectors per block
      for (int v = tid; v < n * kV; v += covf::kThreads) {
        const int r = v / kV, o = 2 * (v % kV);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + r * cov::kBlk + o)),
                     "l"(src + (size_t)ids[r] * cov::kBlk + o)
                     : "memory");
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };

  double ax = 0.0, bx = 0.0, az = 0.0, bz = 0.0;  // inverse Jacobian rows at point q
  double xl[kNl], xd[kNl];                         // l(qx, .), l'(qx, .)
  double tl = 0.0, tm = 0.0, tr = 0.0;
  fetch(0);
  for (int k = 0; k < ntask; k++) {
    const int ei = (int)blockIdx.x + (k / 9) * (int)gridDim.x, b = k % 9;
    const int4 ie = mv.ieng[elems[ei]];
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();  // task k's raw blocks visible; task k - 1 done with every buffer
    fetch(k + 1);
    if (b == 0) {
      if (k == 0) {
#pragma unroll
        for (int i = 0; i < kNl; i++) {
          xl[i] = tl_s[qx * kNl + i];
          xd[i] = td_s[qx * kNl + i];
        }
      }
      tl = tm = tr = 0.0;
      if (ptq) {
        QGeo g;
        if (!quad_geo(mv, dt, ie, q, false, g)) atomicCAS(err, 0, elems[ei] + 1);
        ax = g.dzdeta / g.rjac;
        bx = -g.dzdxi / g.rjac;
        az = -g.dxdeta / g.rjac;
        bz = g.dxdxi / g.rjac;
        const double wq = dt.wts[qx] * dt.wts[qz] * g.rjac;
#pragma unroll
        for (int a = 0; a < 4; a++) wsf_s[a * kNq + q] = dt.sf[4 * q + a] * wq;
      }
    }
    const double *r = rawb + (k & 1) * covf::kRaw;
    const bool two = b < 6;  // Z_l' and the W's beyond (l, l) needed
    // ---- Z stage: task (i, jx)
    if (tid < kNen * kNl) {
      const int i = tid / kNl, jx = tid % kNl;
      double bv[kNl];
#pragma unroll
      for (int je = 0; je < kNl; je++) bv[je] = cov_bval(b, r, i, jx + kNl * je);
      double *ol = zl + (i * kNl + jx) * kNint, *od = zd + (i * kNl + jx) * kNint;
#pragma unroll
      for (int z = 0; z < kNint; z++) {
        double sl = 0.0, sd = 0.0;
#pragma unroll
        for (int je = 0; je < kNl; je++) {
          sl = fma(bv[je], tb.l[z][je], sl);
          sd = fma(bv[je], tb.d[z][je], sd);
        }
        ol[z] = sl;
        if (two) od[z] = sd;
      }
    }
    __syncthreads();
    // ---- W stage: task (ix, jx, qz)
    for (int t = tid; t < covf::kW; t += covf::kThreads) {
      const int z = t % kNint, ixjx = t / kNint, ix = ixjx / kNl, jx = ixjx % kNl;
      double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
#pragma unroll
      for (int ie2 = 0; ie2 < kNl; ie2++) {
        const int zi = ((ix + kNl * ie2) * kNl + jx) * kNint + z;
        const double a = zl[zi];
        const double el = tl_s[z * kNl + ie2], ed = td_s[z * kNl + ie2];
        w0 = fma(el, a, w0);
        if (two) {
          const double c = zd[zi];
          w1 = fma(el, c, w1);
          w2 = fma(ed, a, w2);
          w3 = fma(ed, c, w3);
        }
      }
      wb[t] = w0;
      if (two) {
        wb[covf::kW + t] = w1;
        wb[2 * covf::kW + t] = w2;
        wb[3 * covf::kW + t] = w3;
      }
    }
    __syncthreads();
    // ---- F stage: point q
    if (ptq) {
      const double *W0 = wb, *W1 = wb + covf::kW, *W2 = wb + 2 * covf::kW, *W3 = wb + 3 * covf::kW;
      if (b < 3) {
        const double fxx = cov_fw(W0, qz, xd, xd), fxe = cov_fw(W1, qz, xd, xl);
        const double fee = cov_fw(W3, qz, xl, xl);
        const double xx = ax * ax * fxx + 2.0 * ax * bx * fxe + bx * bx * fee;
        const double zz = az * az * fxx + 2.0 * az * bz * fxe + bz * bz * fee;
        if (b == 0) {
          tl += xx;
          tm += 2.0 * xx + zz;
        } else if (b == 1) {
          tl += zz;
          tm += xx + 2.0 * zz;
        } else {
          tm += xx + zz;
        }
      } else if (b == 3) {
        const double fxx = cov_fw(W0, qz, xd, xd), fxe = cov_fw(W1, qz, xd, xl);
        const double fex = cov_fw(W2, qz, xl, xd), fee = cov_fw(W3, qz, xl, xl);
        tl += ax * az * fxx + ax * bz * fxe + bx * az * fex + bx * bz * fee;  // x^T S z
        tm += az * ax * fxx + az * bx * fxe + bz * ax * fex + bz * bx * fee;  // z^T S x
      } else if (b < 6) {
        const double fxn = cov_fw(W0, qz, xd, xl), fen = cov_fw(W2, qz, xl, xl);
        const double fnx = cov_fw(W0, qz, xl, xd), fne = cov_fw(W1, qz, xl, xl);
        if (b == 4) {
          tl += ax * fxn + bx * fen;  // x^T G1 v
          tm -= ax * fnx + bx * fne;  // v^T G1 x
        } else {
          tl += az * fxn + bz * fen;  // z^T G2 v
          tm -= az * fnx + bz * fne;  // v^T G2 z
        }
      } else {
        const double fnn = cov_fw(W0, qz, xl, xl);
        if (b == 6) {
          tl += fnn;
          tm += 2.0 * fnn;
        } else if (b == 7) {
          tm += fnn;
        } else {
          tr -= fnn;
        }
      }
    }
    if (b == 8) {
      // ---- g_{m, anchor a} += sum_q W_q SF_a(q) T_m(q)
      double v[12];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const double w = ptq ? wsf_s[a * kNq + q] : 0.0;
        v[3 * a + 0] = w * tl;
        v[3 * a + 1] = w * tm;
        v[3 * a + 2] = w * tr;
      }
#pragma unroll
      for (int kk = 0; kk < 12; kk++) {
        double x = v[kk];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[kk] = x;
      }
      if (lane == 0)
        for (int kk = 0; kk < 12; kk++) red[kk][warp] = v[kk];
      __syncthreads();
      if (tid < 12) {
        double x = 0.0;
        for (int w = 0; w < covf::kThreads / 32; w++) x += red[tid][w];
        const int a = tid / 3, m = tid % 3;
        const int anchor = (a == 0 ? ie.x : a == 1 ? ie.y : a == 2 ? ie.z : ie.w) - 1;
        atomicAdd(&grad[(size_t)m * nnpg + anchor], x);
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
static CovFinTabs cov_fin_tables(const Tables &t) {
  // Lagrange basis on the 5 GLL points (the factors of SHL, dshl.f:100-243)
  CovFinTabs tb;
  for (int q = 0; q < kNint; q++) {
    const double x = t.xigll[q];
    for (int i = 0; i < kNl; i++) {
      double v = 1.0, dsum = 0.0;
      for (int k = 0; k < kNl; k++)
        if (k != i) v *= (x - t.xipts[k]) / (t.xipts[i] - t.xipts[k]);
      for (int m = 0; m < kNl; m++) {
        if (m == i) continue;
        double p = 1.0 / (t.xipts[i] - t.xipts[m]);
        for (int k = 0; k < kNl; k++)
          if (k != i && k != m) p *= (x - t.xipts[k]) / (t.xipts[i] - t.xipts[k]);
        dsum += p;
      }
      tb.l[q][i] = v;
      tb.d[q][i] = dsum;
    }
  }
  return tb;
}

// Gather plan of the covariance accumulation for every element outside the
// PML (kernel order): the element's nodes, sorted by first DOF.  An element
// whose 25 nodes are one run of 20 consecutive nodes plus five nodes
// kStrideNodes apart (GENID's numbering of an interior element: its own 20
// nodes, then the column shared with the element numbered before it) takes
// two boxes, a 20-node run and a 5-node strided box; any other element has
// its runs of consecutive nodes covered by boxes of 16, 4 and 1 nodes.  The
// boxes are packed one after the other (8 source rows each) into the
// 9600-byte raw region of a field.  The loader's lanes hold one box each,
// so an element may have at most 32 boxes (set-up refuses a mesh that needs
// more).
static void build_cov_plan(const Ctx *c, const std::vector<int> &elems, std::vector<int2> &ops,
                           std::vector<int> &opptr, std::vector<uint32_t> &node,
                           std::vector<int> &tx) {
  const int n = (int)elems.size();
  const long long ngroups = (long long)c->ndof / 12;  // 4-node groups of the strided view
  opptr.assign(n + 1, 0);
  node.assign((size_t)n * kNen, 0xFFFFFFFFu);
  tx.assign(n, 0);
  ops.clear();
  for (int k = 0; k < n; k++) {
    const int *lme = c->h_lm.data() + (size_t)elems[k] * kNee;
    int ord[kNen], cnt = 0;
    for (int a = 0; a < kNen; a++)
      if (lme[3 * a] > 0) ord[cnt++] = a;
    std::sort(ord, ord + cnt, [&](int x, int y) { return lme[3 * x] < lme[3 * y]; });
    uint32_t off = 0;  // bytes into the field's raw region
    auto box = [&](int code, const int *nodes) {
      const int w = cov::kBoxNodes[code];
      ops.push_back(make_int2(2 * (lme[3 * nodes[0]] - 1), code | (int)(off / 128u) << 8));
      for (int j = 0; j < w; j++)
        node[(size_t)k * kNen + nodes[j]] = (off + (uint32_t)(j * cov::kNodeBytes)) |
                                            ((uint32_t)code << 16);
      off += (uint32_t)(w * cov::kNodeBytes * cov::kG);
    };
    // the two-box form
    bool two = false;
    if (cnt == kNen) {
      for (int r0 = 0; r0 + 20 <= kNen && !two; r0++) {
        bool run = true;
        for (int j = 1; j < 20 && run; j++) run = lme[3 * ord[r0 + j]] == lme[3 * ord[r0]] + 3 * j;
        if (!run) continue;
        int rest[5], nr = 0;
        for (int j = 0; j < kNen; j++)
          if (j < r0 || j >= r0 + 20) rest[nr++] = ord[j];
        bool strided = true;
        for (int j = 1; j < 5 && strided; j++)
          strided = lme[3 * rest[j]] == lme[3 * rest[0]] + 3 * cov::kStrideNodes * j;
        const long long g0 = (long long)(lme[3 * rest[0]] - 1) / 3 / cov::kStrideNodes;
        if (!strided || g0 + 5 > ngroups) continue;
        box(3, ord + r0);
        box(4, rest);
        two = true;
      }
    }
    for (int i = 0; i < cnt && !two;) {
      int len = 1;
      while (i + len < cnt && lme[3 * ord[i + len]] == lme[3 * ord[i]] + 3 * len) len++;
      // boxes of 16, 4 and 1 nodes over the run
      int done = 0;
      while (done < len) {
        const int code = len - done >= 16 ? 0 : len - done >= 4 ? 1 : 2;
        box(code, ord + i + done);
        done += cov::kBoxNodes[code];
      }
      i += len;
    }
    opptr[k + 1] = (int)ops.size();
    tx[k] = (int)(2 * off);
  }
}

// One-time set-up of the covariance gradient: the gather's DOF-layout check,
// the gather plan, the kernels' shared-memory attributes and the FP64
// accumulators (15 x 625 doubles per element outside the PML).  Allocates,
// so it runs outside any stream capture.
cudaError_t prepare_grad_cov(Ctx *c) {
  if (c->d_cov) return cudaSuccess;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return cudaErrorNotSupported;
  c->tmap_encode = fn;
  for (size_t i = 0; i + 2 < c->h_lm.size(); i += 3) {
    const int d = c->h_lm[i];
    const bool ok = d > 0 ? (c->h_lm[i + 1] == d + 1 && c->h_lm[i + 2] == d + 2)
                          : (c->h_lm[i + 1] == 0 && c->h_lm[i + 2] == 0);
    if (!ok) return cudaErrorNotSupported;
  }
  std::vector<int> elems;
  for (int e = 0; e < c->nelem; e++)
    if (c->h_cdomain[e] != 'A') elems.push_back(e);
  std::vector<int2> ops;
  std::vector<int> opptr, tx;
  std::vector<uint32_t> node;
  build_cov_plan(c, elems, ops, opptr, node, tx);
  for (size_t k = 0; k + 1 < opptr.size(); k++)
    if (opptr[k + 1] - opptr[k] > 32) return cudaErrorNotSupported;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_grad_cov, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                cov::kSmemBytes + 128)))
    return e;
  if ((e = cudaFuncSetAttribute(k_grad_cov_fin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                covf::kSmemBytes)))
    return e;
  auto up = [&](void **d, const void *h, size_t bytes) -> cudaError_t {
    cudaError_t r = cudaMalloc(d, bytes ? bytes : 16);
    if (r == cudaSuccess && bytes) r = cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice);
    return r;
  };
  if ((e = up((void **)&c->d_cov_ops, ops.data(), ops.size() * sizeof(int2))) ||
      (e = up((void **)&c->d_cov_opptr, opptr.data(), opptr.size() * sizeof(int))) ||
      (e = up((void **)&c->d_cov_node, node.data(), node.size() * sizeof(uint32_t))) ||
      (e = up((void **)&c->d_cov_tx, tx.data(), tx.size() * sizeof(int))))
    return e;
  if ((e = cudaMalloc((void **)&c->d_cov_exps, sizeof(int) * 2 * kMaxPairs))) return e;
  const size_t n = (size_t)std::max(c->n_nonpml, 1) * cov::kBlocks * cov::kBlk;
  double *d = nullptr;
  if ((e = cudaMalloc(&d, n * sizeof(double)))) return e;
  c->d_cov = d;
  c->cov_pending = false;
  return cudaSuccess;
}

// The TMA views of one launch's fields (CovMaps).  cudaErrorInvalidValue
// for a field pointer off a 16-byte boundary.
static cudaError_t cov_maps(const Ctx *c, const double *u, const double *lam, int rows,
                            CovMaps &maps) {
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(c->tmap_encode);
  const double *base[2] = {u, lam};
  const cuuint32_t estr[3] = {1, 1, 1};
  for (int f = 0; f < 2; f++) {
    if (reinterpret_cast<uintptr_t>(base[f]) % 16) return cudaErrorInvalidValue;
    for (int code = 0; code < cov::kNCodes; code++) {
      CUresult r;
      if (code < 4) {
        const cuuint64_t dim[2] = {(cuuint64_t)2 * c->ndof, (cuuint64_t)rows};
        const cuuint64_t stride[1] = {(cuuint64_t)c->ndof * 16};
        const cuuint32_t boxd[2] = {(cuuint32_t)(6 * cov::kBoxNodes[code]), (cuuint32_t)cov::kG};
        r = encode(&maps.m[f][code], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                   const_cast<double *>(base[f]), dim, stride, boxd, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      } else {
        const cuuint64_t dim[3] = {(cuuint64_t)6 * cov::kStrideNodes, (cuuint64_t)c->ndof / 12,
                                   (cuuint64_t)rows};
        const cuuint64_t stride[2] = {(cuuint64_t)cov::kStrideNodes * cov::kNodeBytes,
                                      (cuuint64_t)c->ndof * 16};
        const cuuint32_t boxd[3] = {6, 5, (cuuint32_t)cov::kG};
        r = encode(&maps.m[f][code], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                   const_cast<double *>(base[f]), dim, stride, boxd, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      }
      if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
  }
  return cudaSuccess;
}

cudaError_t launch_grad_cov(Ctx *c, const PairTable &pt, int npairs, int nsrc, const double *u,
                            const double *lam, cudaStream_t st) {
  if (!c->d_cov) return cudaErrorNotReady;
  if (c->n_nonpml == 0) return cudaSuccess;
  CovMaps maps;
  cudaError_t e = cov_maps(c, u, lam, npairs * nsrc, maps);
  if (e != cudaSuccess) return e;
  // the pairs' field scales
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  if ((e = cudaMemsetAsync(c->d_cov_exps, 0, sizeof(int) * 2 * npairs, st))) return e;
  k_cov_scale<<<dim3(std::max(1, 8 * nsm / npairs), npairs), 256, 0, st>>>(
      reinterpret_cast<const double2 *>(u),
                                                 reinterpret_cast<const double2 *>(lam),
                                                 (long long)nsrc * c->ndof, c->d_cov_exps);
  if ((e = cudaGetLastError())) return e;
  CovArgs ga;
  ga.exps = c->d_cov_exps;
  ga.npairs = npairs;
  ga.nsrc = nsrc;
  ga.ndof = c->ndof;
  ga.n_elem = c->n_nonpml;
  ga.add = c->cov_pending ? 1 : 0;
  ga.inject = c->wait_inject;
  ga.spin = c->wait_limit > 0 ? c->wait_limit : kTcSpinCycles;
  CovPlan plan{c->d_cov_ops, c->d_cov_opptr, c->d_cov_node, c->d_cov_tx};
  const int grid = std::min(nsm, c->n_nonpml);
  k_grad_cov<<<grid, cov::kThreads, cov::kSmemBytes + 128, st>>>(maps, ga, plan, pt, c->d_cov,
                                                                 c->d_err);
  e = cudaGetLastError();
  if (e == cudaSuccess) c->cov_pending = true;
  return e;
}

cudaError_t launch_grad_cov_fin(Ctx *c, double *grad, cudaStream_t st) {
  if (!c->d_cov) return cudaErrorNotReady;
  if (!c->cov_pending || c->n_nonpml == 0) return cudaSuccess;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  const int grid = std::min(3 * nsm, c->n_nonpml);
  k_grad_cov_fin<<<grid, covf::kThreads, covf::kSmemBytes, st>>>(
      c->mv, c->dt, c->n_nonpml, c->nnpg, c->d_nonpml, c->d_cov, cov_fin_tables(c->tab), grad,
      c->d_err);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) c->cov_pending = false;
  return e;
}

}  // namespace fem25
