// Batched assembly of many (omega, py) systems of one mesh.
//
// For every non-PML element the KM25ISOQ matrix (estiff25.f:64-154) is affine
// in (omega^2, omega*py, (omega*py)^2):
//   A(i,j) = delta_ij (-omega^2 M_rho + (omega py)^2 M_i) + K0_ij + i omega py K1_ij
// with real K0 on the (1,1),(1,3),(2,2),(3,1),(3,3) component blocks, real K1
// on (1,2),(2,1),(2,3),(3,2), M_1 = M_3 = int mu N_a N_b, M_2 = int (lambda+2mu)
// N_a N_b.  The PML elements (CM25ISOQ, estiff25.f:235-332) share the mass
// part and add CE0(omega) + omega py CE1(omega) with complex coefficients.
// The basis is summed once per mesh into 3x3 node blocks of the CSR (12 reals
// per block); the streaming kernel then reads each block's basis once per
// pass and writes it for B systems: an HBM-write-bound stream.
#include <cstdlib>

#include "ctx.cuh"
#include "kcommon.cuh"

namespace fem25 {

cudaError_t scan_counts(const int *count, int *ptr, long long n, cudaStream_t st);
__global__ void k_sort_lists(long long n, const int *__restrict__ ptr, int *__restrict__ list,
                             int *__restrict__ err);

// basis slots per block
enum { B_K11 = 0, B_K13, B_K22, B_K31, B_K33, B_K12, B_K21, B_K23, B_K32, B_MRHO, B_MMU, B_ML2M, B_N };

constexpr int kElemThreads = 640;

// Per element node pair: the 12 basis integrals over the 13x13 rule.
// PML elements contribute their (omega-independent) mass integrals only.
__global__ void __launch_bounds__(kElemThreads, 1)
    k_elem_basis(MeshView mv, DevTables dt, double *__restrict__ ebasis, int *__restrict__ err) {
  extern __shared__ double sm[];
  double *shx = sm, *shz = sm + kNq * kNen, *shn = sm + 2 * kNq * kNen, *qc = sm + 3 * kNq * kNen;
  const int e = blockIdx.x, t = threadIdx.x;
  const int4 ie = mv.ieng[e];
  const bool pml = mv.cdomain[e] == 'A';
  if (t < kNq) {
    const int q = t, intx = q % kNint, intz = q / kNint;
    QGeo g;
    if (!quad_geo(mv, dt, ie, q, false, g)) atomicCAS(err, 0, e + 1);
    double *c = qc + 8 * q;
    c[0] = g.dxdxi; c[1] = g.dxdeta; c[2] = g.dzdxi; c[3] = g.dzdeta; c[4] = g.rjac;
    double w = dt.wts[intx] * dt.wts[intz] * g.rjac;
    c[5] = g.lam * w;
    c[6] = g.mu * w;
    c[7] = g.rho * w;
  }
  __syncthreads();
  for (int idx = t; idx < kNq * kNen; idx += kElemThreads) {
    const int q = idx / kNen;
    const double *c = qc + 8 * q;
    const double *sl = dt.shl + 3 * (size_t)idx;
    shx[idx] = (sl[0] * c[3] - sl[1] * c[2]) / c[4];
    shz[idx] = -(sl[0] * c[1] - sl[1] * c[0]) / c[4];
    shn[idx] = sl[2];
  }
  __syncthreads();
  if (t >= kNab) return;
  const int a = t / kNen, b = t % kNen;
  double acc[B_N];
#pragma unroll
  for (int k = 0; k < B_N; k++) acc[k] = 0.0;
  for (int q = 0; q < kNq; q++) {
    const double *c = qc + 8 * q;
    const double lam = c[5], mu = c[6], rhow = c[7], c11 = lam + 2.0 * mu;
    const double pa = shn[q * kNen + a], pax = shx[q * kNen + a], paz = shz[q * kNen + a];
    const double pb = shn[q * kNen + b], pbx = shx[q * kNen + b], pbz = shz[q * kNen + b];
    const double nn = pa * pb;
    acc[B_MRHO] += nn * rhow;
    acc[B_MMU] += nn * mu;
    acc[B_ML2M] += nn * c11;
    if (!pml) {
      acc[B_K11] += pax * c11 * pbx + paz * mu * pbz;
      acc[B_K13] += pax * lam * pbz + paz * mu * pbx;
      acc[B_K22] += pax * mu * pbx + paz * mu * pbz;
      acc[B_K31] += paz * lam * pbx + pax * mu * pbz;
      acc[B_K33] += paz * c11 * pbz + pax * mu * pbx;
      acc[B_K12] += -(lam * pax * pb - mu * pa * pbx);
      acc[B_K21] += (lam * pa * pbx - mu * pax * pb);
      acc[B_K23] += (lam * pa * pbz - mu * paz * pb);
      acc[B_K32] += -(lam * paz * pb - mu * pa * pbz);
    }
  }
  double *o = ebasis + ((size_t)e * kNab + t) * B_N;
#pragma unroll
  for (int k = 0; k < B_N; k++) o[k] = acc[k];
}

// Per PML element node pair at one omega: the 9 complex CE coefficients
// (CE0 on the (1,1),(1,3),(2,2),(3,1),(3,3) blocks, CE1 -- the coefficient of
// omega*py -- on the others), entry k = 3i+j.
__global__ void __launch_bounds__(kElemThreads, 1)
    k_elem_pml(MeshView mv, DevTables dt, const int *__restrict__ pml_elems, PmlParams pp,
               double logr, double2 *__restrict__ pemat, int *__restrict__ err) {
  extern __shared__ double sm[];
  double *shx = sm, *shz = sm + kNq * kNen, *qc = sm + 2 * kNq * kNen;
  const int pe = blockIdx.x, e = pml_elems[pe], t = threadIdx.x;
  const int4 ie = mv.ieng[e];
  if (t < kNq) {
    const int q = t, intx = q % kNint, intz = q / kNint;
    QGeo g;
    if (!quad_geo(mv, dt, ie, q, true, g)) atomicCAS(err, 0, e + 1);
    dcx ex = dcx{1.0, 0.0}, ez = dcx{1.0, 0.0};
    if (g.xdep > 2.22e-16)
      ex = zdampfn(g.xdep, g.vel, pp.xwidth, pp.dmax, logr, pp.kappa, pp.fcent, pp.omega);
    if (g.zdep > 2.22e-16)
      ez = zdampfn(g.zdep, g.vel, pp.zwidth, pp.dmax, logr, pp.kappa, pp.fcent, pp.omega);
    double *c = qc + 11 * q;
    c[0] = g.dxdxi; c[1] = g.dxdeta; c[2] = g.dzdxi; c[3] = g.dzdeta; c[4] = g.rjac;
    double w = dt.wts[intx] * dt.wts[intz] * g.rjac;
    c[5] = g.lam * w;
    c[6] = g.mu * w;
    c[7] = ex.re; c[8] = ex.im; c[9] = ez.re; c[10] = ez.im;
  }
  __syncthreads();
  for (int idx = t; idx < kNq * kNen; idx += kElemThreads) {
    const int q = idx / kNen;
    const double *c = qc + 11 * q;
    const double *sl = dt.shl + 3 * (size_t)idx;
    shx[idx] = (sl[0] * c[3] - sl[1] * c[2]) / c[4];
    shz[idx] = -(sl[0] * c[1] - sl[1] * c[0]) / c[4];
  }
  __syncthreads();
  if (t >= kNab) return;
  const int a = t / kNen, b = t % kNen;
  dcx acc[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = dcx{0.0, 0.0};
  for (int q = 0; q < kNq; q++) {
    const double *c = qc + 11 * q;
    const double lam = c[5], mu = c[6], c11 = lam + 2.0 * mu;
    const dcx ex = dcx{c[7], c[8]}, ez = dcx{c[9], c[10]};
    const double pa = dt.shl[3 * (q * kNen + a) + 2], pb = dt.shl[3 * (q * kNen + b) + 2];
    const dcx pax = dcx{shx[q * kNen + a] * ex.re, shx[q * kNen + a] * ex.im};
    const dcx paz = dcx{shz[q * kNen + a] * ez.re, shz[q * kNen + a] * ez.im};
    const dcx pbx = dcx{shx[q * kNen + b] * ex.re, shx[q * kNen + b] * ex.im};
    const dcx pbz = dcx{shz[q * kNen + b] * ez.re, shz[q * kNen + b] * ez.im};
    // CE0 blocks
    dcx xx = zmul(pax, pbx), zz = zmul(paz, pbz), xz = zmul(pax, pbz), zx = zmul(paz, pbx);
    acc[0] = zadd(acc[0], dcx{c11 * xx.re + mu * zz.re, c11 * xx.im + mu * zz.im});
    acc[2] = zadd(acc[2], dcx{lam * xz.re + mu * zx.re, lam * xz.im + mu * zx.im});
    acc[4] = zadd(acc[4], dcx{mu * xx.re + mu * zz.re, mu * xx.im + mu * zz.im});
    acc[6] = zadd(acc[6], dcx{lam * zx.re + mu * xz.re, lam * zx.im + mu * xz.im});
    acc[8] = zadd(acc[8], dcx{c11 * zz.re + mu * xx.re, c11 * zz.im + mu * xx.im});
    // CE1 blocks: i * (...)
    dcx t12 = dcx{-(lam * pax.re * pb - mu * pa * pbx.re), -(lam * pax.im * pb - mu * pa * pbx.im)};
    dcx t21 = dcx{lam * pa * pbx.re - mu * pax.re * pb, lam * pa * pbx.im - mu * pax.im * pb};
    dcx t23 = dcx{lam * pa * pbz.re - mu * paz.re * pb, lam * pa * pbz.im - mu * paz.im * pb};
    dcx t32 = dcx{-(lam * paz.re * pb - mu * pa * pbz.re), -(lam * paz.im * pb - mu * pa * pbz.im)};
    acc[1] = zadd(acc[1], dcx{-t12.im, t12.re});
    acc[3] = zadd(acc[3], dcx{-t21.im, t21.re});
    acc[5] = zadd(acc[5], dcx{-t23.im, t23.re});
    acc[7] = zadd(acc[7], dcx{-t32.im, t32.re});
  }
  double2 *o = pemat + ((size_t)pe * kNab + t) * 9;
#pragma unroll
  for (int k = 0; k < 9; k++) o[k] = make_double2(acc[k].re, acc[k].im);
}

// block id of element node pair (a,b): position of node B in block row A
__device__ __forceinline__ long long find_block(const long long *brptr, const int *bcol, int A,
                                                int B) {
  long long lo = brptr[A], hi = brptr[A + 1] - 1;
  while (lo <= hi) {
    long long mid = (lo + hi) >> 1;
    int v = bcol[mid];
    if (v == B) return mid;
    if (v < B) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

__global__ void k_map_blocks(int nelem, const int *__restrict__ lm, const long long *__restrict__ brptr,
                             const int *__restrict__ bcol, int *__restrict__ count,
                             const int *__restrict__ ptr, int *__restrict__ cursor,
                             int *__restrict__ list, int pass, int *__restrict__ err) {
  long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)nelem * kNab) return;
  int e = (int)(gid / kNab), ab = (int)(gid % kNab);
  int a = ab / kNen, b = ab % kNen;
  int ra = lm[(size_t)e * kNee + 3 * a], rb = lm[(size_t)e * kNee + 3 * b];
  if (ra <= 0 || rb <= 0) return;
  long long blk = find_block(brptr, bcol, (ra - 1) / 3, (rb - 1) / 3);
  if (blk < 0) {
    atomicCAS(err, 0, e + 1);
    return;
  }
  if (pass == 0) {
    atomicAdd(&count[blk], 1);
  } else {
    int slot = atomicAdd(&cursor[blk], 1);
    list[ptr[blk] + slot] = (int)gid;
  }
}

__global__ void k_gather_basis(long long nblocks, const int *__restrict__ ptr,
                               const int *__restrict__ list, const double *__restrict__ ebasis,
                               double *__restrict__ basis) {
  long long blk = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= nblocks) return;
  double acc[B_N];
#pragma unroll
  for (int k = 0; k < B_N; k++) acc[k] = 0.0;
  for (int i = ptr[blk]; i < ptr[blk + 1]; i++) {
    const double *s = ebasis + (size_t)list[i] * B_N;
#pragma unroll
    for (int k = 0; k < B_N; k++) acc[k] += s[k];
  }
#pragma unroll
  for (int k = 0; k < B_N; k++) basis[(size_t)k * nblocks + blk] = acc[k];
}

// PML structure: count the PML contributors of every block
__global__ void k_pml_count(long long nblocks, const int *__restrict__ ptr,
                            const int *__restrict__ list, const char *__restrict__ cdomain,
                            int *__restrict__ pcount, int *__restrict__ isp) {
  long long blk = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= nblocks) return;
  int n = 0;
  for (int i = ptr[blk]; i < ptr[blk + 1]; i++)
    if (cdomain[list[i] / kNab] == 'A') n++;
  pcount[blk] = n;
  isp[blk] = n > 0 ? 1 : 0;
}

__global__ void k_pml_fill(long long nblocks, const int *__restrict__ ptr,
                           const int *__restrict__ list, const char *__restrict__ cdomain,
                           const int *__restrict__ isp_scan, const int *__restrict__ pml_local,
                           const int *__restrict__ pcount_scan_by_pblk, int *__restrict__ pml_idx,
                           int *__restrict__ plist) {
  long long blk = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= nblocks) return;
  bool has = false;
  for (int i = ptr[blk]; i < ptr[blk + 1]; i++)
    if (cdomain[list[i] / kNab] == 'A') has = true;
  if (!has) {
    pml_idx[blk] = -1;
    return;
  }
  int pb = isp_scan[blk];
  pml_idx[blk] = pb;
  int o = pcount_scan_by_pblk[pb];
  for (int i = ptr[blk]; i < ptr[blk + 1]; i++) {
    int id = list[i], e = id / kNab;
    if (cdomain[e] == 'A') plist[o++] = pml_local[e] * kNab + id % kNab;
  }
}

__global__ void k_compact_counts(long long nblocks, const int *__restrict__ pcount,
                                 const int *__restrict__ isp_scan, int *__restrict__ pcount_c) {
  long long blk = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk >= nblocks) return;
  if (pcount[blk] > 0) pcount_c[isp_scan[blk]] = pcount[blk];
}

__global__ void k_gather_pml(long long npblk, const int *__restrict__ pptr,
                             const int *__restrict__ plist, const double2 *__restrict__ pemat,
                             double2 *__restrict__ delta) {
  long long pb = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (pb >= npblk) return;
  double2 acc[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = make_double2(0.0, 0.0);
  for (int i = pptr[pb]; i < pptr[pb + 1]; i++) {
    const double2 *s = pemat + (size_t)plist[i] * 9;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      acc[k].x += s[k].x;
      acc[k].y += s[k].y;
    }
  }
#pragma unroll
  for (int k = 0; k < 9; k++) delta[pb * 9 + k] = acc[k];
}

// ---------------------------------------------------------------------------
// the streaming kernel
// ---------------------------------------------------------------------------
constexpr int kStreamThreads = 256;

__device__ __forceinline__ void st_cs(double2 *p, double2 v) {
  asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}

// basis slot of CSR entry (i, j) of a 3x3 block
__device__ __constant__ int kEntrySlot[9] = {B_K11, B_K12, B_K13, B_K21, B_K22,
                                             B_K23, B_K31, B_K32, B_K33};

// Per-entry "primary" basis value in CSR order (K0_ij on the real entries,
// K1_ij on the entries that carry i*omega*py) and a packed descriptor
// desc = block << 4 | i << 2 | j.  One warp per block row: the three CSR rows
// of a node are contiguous ([9 b0, 9 b1)), row i holds 3 deg entries, entry r
// of a row is block b0 + r/3, component r%3.
__global__ void k_build_prim(int nbrow, const long long *__restrict__ brptr,
                             const double *__restrict__ basis, long long nblocks,
                             double *__restrict__ prim, unsigned *__restrict__ desc) {
  const int lane = threadIdx.x & 31;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  for (long long A = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; A < nbrow; A += nwarp) {
    const long long b0 = brptr[A];
    const int deg = (int)(brptr[A + 1] - b0), rl = 3 * deg;
    for (int nl = lane; nl < 9 * deg; nl += 32) {
      const int i = (nl >= rl) + (nl >= 2 * rl);
      const int r = nl - i * rl, t = r / 3, j = r - 3 * t;
      prim[9 * b0 + nl] = basis[(size_t)kEntrySlot[3 * i + j] * nblocks + b0 + t];
      desc[9 * b0 + nl] = ((unsigned)(b0 + t) << 4) | (unsigned)(i << 2) | (unsigned)j;
    }
  }
}

// One launch writes systems [s0, s1) (at most kMaxPass, each to its own ring
// slot).  Grid-stride over the CSR entries: each thread takes UNR entries
// (n, n + G, ...), issues all their loads (primary value and descriptor,
// then the block's mass terms and PML index) before any store, and writes
// each entry for every system of the launch.  Consecutive threads hold
// consecutive entries, so each warp store writes 512 contiguous bytes.
// Launches that reuse ring slots are ordered by the stream.
template <int UNR>
__global__ void __launch_bounds__(kStreamThreads)
    k_stream(long long nzero, const double *__restrict__ prim, const unsigned *__restrict__ desc,
             const double *__restrict__ basis, long long nblocks, const int *__restrict__ pml_idx,
             const double2 *__restrict__ pml_delta, long long npblk, SysTable tab,
             int s0, int s1, double *__restrict__ ring, long long stride, int nslots) {
  __shared__ SysParam sp[kMaxPass];
  __shared__ double2 *outp[kMaxPass];
  const int ns = s1 - s0;
  if (threadIdx.x < ns) {
    sp[threadIdx.x] = tab.s[threadIdx.x];
    outp[threadIdx.x] =
        reinterpret_cast<double2 *>(ring + (size_t)((s0 + threadIdx.x) % nslots) * stride);
  }
  __syncthreads();
  const long long G = (long long)gridDim.x * blockDim.x;
  const double *mrho = basis + (size_t)B_MRHO * nblocks;
  const double *mmu = basis + (size_t)B_MMU * nblocks;
  const double *ml2m = basis + (size_t)B_ML2M * nblocks;
  for (long long n0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; n0 < nzero; n0 += UNR * G) {
    double p[UNR], mr[UNR], mc[UNR];
    unsigned d[UNR];
    int pidx[UNR];
#pragma unroll
    for (int u = 0; u < UNR; u++) {
      const long long n = n0 + u * G;
      d[u] = 0u;
      p[u] = 0.0;
      if (n < nzero) {
        p[u] = __ldcs(prim + n);
        d[u] = __ldcs(desc + n);
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; u++) {
      const unsigned blk = d[u] >> 4, i = (d[u] >> 2) & 3u, j = d[u] & 3u;
      mr[u] = 0.0;
      mc[u] = 0.0;
      if (i == j) {
        mr[u] = mrho[blk];
        mc[u] = (i == 1u) ? ml2m[blk] : mmu[blk];
      }
      pidx[u] = pml_idx[blk];
    }
    for (int k = 0; k < ns; k++) {
      const double w2 = sp[k].w2, wpy = sp[k].wpy, wpy2 = wpy * wpy;
      const int slot = sp[k].pml_slot;
      double2 *o = outp[k];
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        const long long n = n0 + u * G;
        if (n >= nzero) continue;
        const unsigned i = (d[u] >> 2) & 3u, j = d[u] & 3u;
        const bool odd = (i + j) & 1u;
        double2 v;
        if (odd) v = make_double2(0.0, wpy * p[u]);
        else v = make_double2(p[u] - w2 * mr[u] + wpy2 * mc[u], 0.0);  // mr = mc = 0 off the diagonal
        if (pidx[u] >= 0) {
          const double2 dv = pml_delta[((size_t)slot * npblk + pidx[u]) * 9 + 3 * i + j];
          const double f = odd ? wpy : 1.0;
          v.x += f * dv.x;
          v.y += f * dv.y;
        }
        st_cs(o + n, v);
      }
    }
  }
}

// Same as k_stream<1>, software-pipelined over the grid-stride loop: while
// the stores of entry n are issued, the descriptor/primary loads of n+2G and
// the block loads (mass terms, PML index) of n+G are already in flight.
struct EntryIn {
  double p, mr, mc;
  unsigned d;
  int pidx;
};

__global__ void __launch_bounds__(kStreamThreads)
    k_stream_pipe(long long nzero, const double *__restrict__ prim, const unsigned *__restrict__ desc,
                  const double *__restrict__ basis, long long nblocks, const int *__restrict__ pml_idx,
                  const double2 *__restrict__ pml_delta, long long npblk,
                  SysTable tab, int s0, int s1, double *__restrict__ ring,
                  long long stride, int nslots) {
  __shared__ SysParam sp[kMaxPass];
  __shared__ double2 *outp[kMaxPass];
  const int ns = s1 - s0;
  if (threadIdx.x < ns) {
    sp[threadIdx.x] = tab.s[threadIdx.x];
    outp[threadIdx.x] =
        reinterpret_cast<double2 *>(ring + (size_t)((s0 + threadIdx.x) % nslots) * stride);
  }
  __syncthreads();
  const long long G = (long long)gridDim.x * blockDim.x;
  const double *mrho = basis + (size_t)B_MRHO * nblocks;
  const double *mmu = basis + (size_t)B_MMU * nblocks;
  const double *ml2m = basis + (size_t)B_ML2M * nblocks;
  auto ld1 = [&](long long n, double &p, unsigned &d) {
    p = 0.0;
    d = 0u;
    if (n < nzero) {
      p = __ldcs(prim + n);
      d = __ldcs(desc + n);
    }
  };
  auto ld2 = [&](unsigned d, double &mr, double &mc, int &pidx) {
    const unsigned blk = d >> 4, i = (d >> 2) & 3u, j = d & 3u;
    mr = 0.0;
    mc = 0.0;
    if (i == j) {
      mr = mrho[blk];
      mc = (i == 1u) ? ml2m[blk] : mmu[blk];
    }
    pidx = pml_idx[blk];
  };
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double pa, pb, mra, mca;
  unsigned da, db;
  int pia;
  ld1(n, pa, da);
  ld1(n + G, pb, db);
  ld2(da, mra, mca, pia);
  for (; n < nzero; n += G) {
    double pc;
    unsigned dc;
    ld1(n + 2 * G, pc, dc);        // two ahead
    double mrb, mcb;
    int pib;
    ld2(db, mrb, mcb, pib);         // one ahead
    const unsigned i = (da >> 2) & 3u, j = da & 3u;
    const bool odd = (i + j) & 1u;
    for (int k = 0; k < ns; k++) {
      const double w2 = sp[k].w2, wpy = sp[k].wpy;
      double2 v;
      if (odd) v = make_double2(0.0, wpy * pa);
      else v = make_double2(pa - w2 * mra + (wpy * wpy) * mca, 0.0);
      if (pia >= 0) {
        const double2 dv = pml_delta[((size_t)sp[k].pml_slot * npblk + pia) * 9 + 3 * i + j];
        const double f = odd ? wpy : 1.0;
        v.x += f * dv.x;
        v.y += f * dv.y;
      }
      st_cs(outp[k] + n, v);
    }
    pa = pb; da = db; mra = mrb; mca = mcb; pia = pib;
    pb = pc; db = dc;
  }
}

// TMA variant: each CTA computes a chunk of T consecutive entries for all
// systems of the launch into a shared-memory staging buffer (one contiguous
// T*16-byte run per system), then one thread hands every run to the TMA unit
// with cp.async.bulk.global.shared::cta (untiled bulk store: 16-byte aligned
// addresses, sizes a multiple of 16).  Two staging buffers alternate, so the
// bulk stores of chunk c drain while chunk c+1 is computed.
__device__ __forceinline__ void bulk_store(void *gdst, const void *ssrc, unsigned bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(ssrc);
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(s),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <int T>
__global__ void __launch_bounds__(T)
    k_stream_tma(long long nzero, const double *__restrict__ prim, const unsigned *__restrict__ desc,
                 const double *__restrict__ basis, long long nblocks, const int *__restrict__ pml_idx,
                 const double2 *__restrict__ pml_delta, long long npblk,
                 SysTable tab, int s0, int s1, double *__restrict__ ring,
                 long long stride, int nslots) {
  extern __shared__ __align__(128) double2 stage[];  // [2][kMaxPass][T]
  __shared__ SysParam sp[kMaxPass];
  __shared__ double2 *outp[kMaxPass];
  const int ns = s1 - s0;
  if (threadIdx.x < ns) {
    sp[threadIdx.x] = tab.s[threadIdx.x];
    outp[threadIdx.x] =
        reinterpret_cast<double2 *>(ring + (size_t)((s0 + threadIdx.x) % nslots) * stride);
  }
  __syncthreads();
  const double *mrho = basis + (size_t)B_MRHO * nblocks;
  const double *mmu = basis + (size_t)B_MMU * nblocks;
  const double *ml2m = basis + (size_t)B_ML2M * nblocks;
  const long long nchunk = (nzero + T - 1) / T;
  int it = 0;
  for (long long c = blockIdx.x; c < nchunk; c += gridDim.x, it++) {
    double2 *buf = stage + (size_t)(it & 1) * kMaxPass * T;
    if (it >= 2) {
      // the bulk stores issued from this buffer two chunks ago must have
      // finished reading it
      if (threadIdx.x == 0) bulk_wait_read1();
      __syncthreads();
    }
    const long long n0 = c * T, n = n0 + threadIdx.x;
    if (n < nzero) {
      const double p = __ldcs(prim + n);
      const unsigned d = __ldcs(desc + n);
      const unsigned blk = d >> 4, i = (d >> 2) & 3u, j = d & 3u;
      double mr = 0.0, mc = 0.0;
      if (i == j) {
        mr = mrho[blk];
        mc = (i == 1u) ? ml2m[blk] : mmu[blk];
      }
      const int pidx = pml_idx[blk];
      const bool odd = (i + j) & 1u;
      for (int k = 0; k < ns; k++) {
        const double w2 = sp[k].w2, wpy = sp[k].wpy;
        double2 v;
        if (odd) v = make_double2(0.0, wpy * p);
        else v = make_double2(p - w2 * mr + (wpy * wpy) * mc, 0.0);
        if (pidx >= 0) {
          const double2 dv = pml_delta[((size_t)sp[k].pml_slot * npblk + pidx) * 9 + 3 * i + j];
          const double f = odd ? wpy : 1.0;
          v.x += f * dv.x;
          v.y += f * dv.y;
        }
        buf[k * T + threadIdx.x] = v;
      }
    }
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long cnt = min((long long)T, nzero - n0);
      for (int k = 0; k < ns; k++) bulk_store(outp[k] + n0, buf + k * T, (unsigned)(cnt * 16));
      bulk_commit();
    }
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// Staging-ring variant: a CTA of T threads computes a chunk of T consecutive
// entries and hands it to the TMA unit one system at a time (one T*16-byte
// bulk store per system) through a ring of NB shared-memory buffers, so the
// shared memory per CTA stays at NB*T*16 bytes whatever the number of systems
// and the SM keeps enough resident warps to hide the input loads; the inputs
// of the CTA's next chunk are loaded before the stores of the current one.
// Each system's store is its own bulk group: before a buffer is refilled,
// thread 0 waits until at most NB-1 groups still read shared memory.
template <int T, int NB>
__global__ void __launch_bounds__(T)
    k_stream_ring(long long nzero, const double *__restrict__ prim, const unsigned *__restrict__ desc,
                  const double *__restrict__ basis, long long nblocks, const int *__restrict__ pml_idx,
                  const double2 *__restrict__ pml_delta, long long npblk, SysTable tab, int s0,
                  int s1, double *__restrict__ ring, long long stride, int nslots) {
  extern __shared__ __align__(128) double2 stage[];  // [NB][T]
  __shared__ SysParam sp[kMaxPass];
  __shared__ double2 *outp[kMaxPass];
  const int ns = s1 - s0;
  if (threadIdx.x < ns) {
    sp[threadIdx.x] = tab.s[threadIdx.x];
    outp[threadIdx.x] =
        reinterpret_cast<double2 *>(ring + (size_t)((s0 + threadIdx.x) % nslots) * stride);
  }
  __syncthreads();
  const double *mrho = basis + (size_t)B_MRHO * nblocks;
  const double *mmu = basis + (size_t)B_MMU * nblocks;
  const double *ml2m = basis + (size_t)B_ML2M * nblocks;
  auto load = [&](long long n, double &p, unsigned &d, double &mr, double &mc, int &pidx) {
    p = 0.0;
    d = 0u;
    mr = 0.0;
    mc = 0.0;
    pidx = -1;
    if (n >= nzero) return;
    p = __ldcs(prim + n);
    d = __ldcs(desc + n);
    const unsigned blk = d >> 4, i = (d >> 2) & 3u, j = d & 3u;
    if (i == j) {
      mr = mrho[blk];
      mc = (i == 1u) ? ml2m[blk] : mmu[blk];
    }
    pidx = pml_idx[blk];
  };
  const long long nchunk = (nzero + T - 1) / T;
  long long c = blockIdx.x;
  double p, mr, mc;
  unsigned d;
  int pidx;
  load(c * T + threadIdx.x, p, d, mr, mc, pidx);
  int q = 0;  // running buffer count
  for (; c < nchunk; c += gridDim.x) {
    const long long n0 = c * T, n = n0 + threadIdx.x;
    double p2, mr2, mc2;
    unsigned d2;
    int pidx2;
    load((c + gridDim.x) * T + threadIdx.x, p2, d2, mr2, mc2, pidx2);  // next chunk
    const unsigned i = (d >> 2) & 3u, j = d & 3u;
    const bool odd = (i + j) & 1u;
    const unsigned cnt = (unsigned)min((long long)T, nzero - n0);
    for (int k = 0; k < ns; k++, q++) {
      double2 *buf = stage + (size_t)(q % NB) * T;
      if (q >= NB && threadIdx.x == 0) bulk_wait_read<NB - 1>();
      __syncthreads();
      if (n < nzero) {
        const double w2 = sp[k].w2, wpy = sp[k].wpy;
        double2 v;
        if (odd) v = make_double2(0.0, wpy * p);
        else v = make_double2(p - w2 * mr + (wpy * wpy) * mc, 0.0);
        if (pidx >= 0) {
          const double2 dv = pml_delta[((size_t)sp[k].pml_slot * npblk + pidx) * 9 + 3 * i + j];
          const double f = odd ? wpy : 1.0;
          v.x += f * dv.x;
          v.y += f * dv.y;
        }
        buf[threadIdx.x] = v;
      }
      fence_async_smem();
      __syncthreads();
      if (threadIdx.x == 0) {
        bulk_store(outp[k] + n0, buf, cnt * 16u);
        bulk_commit();
      }
    }
    p = p2;
    d = d2;
    mr = mr2;
    mc = mc2;
    pidx = pidx2;
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// Large-ring staging ring: as k_stream_ring, but one launch takes up to
// kMaxBatch systems (their parameters a 24 KB __grid_constant__ argument), so
// with a ring of more than 16 slots each CTA reads its chunk's basis entries
// once per min(nslots, 1024) systems instead of once per 16.  A launch never
// holds more systems than the ring has slots: two systems of one launch in the
// same slot would overwrite each other in L2, and most of them would never
// reach memory.
template <int T, int NB>
__global__ void __launch_bounds__(T)
    k_stream_big(long long nzero, const double *__restrict__ prim, const unsigned *__restrict__ desc,
                 const double *__restrict__ basis, long long nblocks, const int *__restrict__ pml_idx,
                 const double2 *__restrict__ pml_delta, long long npblk,
                 const __grid_constant__ SysTableBig tab, int s0, int s1,
                 double *__restrict__ ring, long long stride, int nslots) {
  extern __shared__ __align__(128) double2 stage[];  // [NB][T]
  const int ns = s1 - s0;  // <= nslots
  const double *mrho = basis + (size_t)B_MRHO * nblocks;
  const double *mmu = basis + (size_t)B_MMU * nblocks;
  const double *ml2m = basis + (size_t)B_ML2M * nblocks;
  auto load = [&](long long n, double &p, unsigned &d, double &mr, double &mc, int &pidx) {
    p = 0.0;
    d = 0u;
    mr = 0.0;
    mc = 0.0;
    pidx = -1;
    if (n >= nzero) return;
    p = __ldcs(prim + n);
    d = __ldcs(desc + n);
    const unsigned blk = d >> 4, i = (d >> 2) & 3u, j = d & 3u;
    if (i == j) {
      mr = mrho[blk];
      mc = (i == 1u) ? ml2m[blk] : mmu[blk];
    }
    pidx = pml_idx[blk];
  };
  const long long nchunk = (nzero + T - 1) / T;
  long long c = blockIdx.x;
  double p, mr, mc;
  unsigned d;
  int pidx;
  load(c * T + threadIdx.x, p, d, mr, mc, pidx);
  int q = 0;  // running buffer count
  for (; c < nchunk; c += gridDim.x) {
    const long long n0 = c * T, n = n0 + threadIdx.x;
    double p2, mr2, mc2;
    unsigned d2;
    int pidx2;
    load((c + gridDim.x) * T + threadIdx.x, p2, d2, mr2, mc2, pidx2);  // next chunk
    const unsigned i = (d >> 2) & 3u, j = d & 3u;
    const bool odd = (i + j) & 1u;
    const unsigned cnt = (unsigned)min((long long)T, nzero - n0);
    for (int k = 0; k < ns; k++, q++) {
      double2 *buf = stage + (size_t)(q % NB) * T;
      if (q >= NB && threadIdx.x == 0) bulk_wait_read<NB - 1>();
      __syncthreads();
      if (n < nzero) {
        const SysParam &sy = tab.s[k];
        const double w2 = sy.w2, wpy = sy.wpy;
        double2 v;
        if (odd) v = make_double2(0.0, wpy * p);
        else v = make_double2(p - w2 * mr + (wpy * wpy) * mc, 0.0);
        if (pidx >= 0) {
          const double2 dv = pml_delta[((size_t)sy.pml_slot * npblk + pidx) * 9 + 3 * i + j];
          const double f = odd ? wpy : 1.0;
          v.x += f * dv.x;
          v.y += f * dv.y;
        }
        buf[threadIdx.x] = v;
      }
      fence_async_smem();
      __syncthreads();
      if (threadIdx.x == 0) {
        double2 *o = reinterpret_cast<double2 *>(ring + (size_t)((s0 + k) % nslots) * stride);
        bulk_store(o + n0, buf, cnt * 16u);
        bulk_commit();
      }
    }
    p = p2;
    d = d2;
    mr = mr2;
    mc = mc2;
    pidx = pidx2;
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static size_t basis_smem() { return sizeof(double) * (3 * kNq * kNen + 8 * kNq); }
static size_t pml_smem() { return sizeof(double) * (2 * kNq * kNen + 11 * kNq); }

cudaError_t build_batch_structures(Ctx *c, cudaStream_t st) {
  cudaError_t e;
  const long long nb = c->bcsr.nblocks;
  int *d_bcol = nullptr, *d_count = nullptr, *d_cursor = nullptr;
  if ((e = cudaMalloc(&c->d_brptr, sizeof(long long) * (c->bcsr.nbrow + 1)))) return e;
  if ((e = cudaMalloc(&c->d_brow, sizeof(int) * nb))) return e;
  if ((e = cudaMallocAsync(&d_bcol, sizeof(int) * nb, st))) return e;
  cudaMemcpyAsync(c->d_brptr, c->bcsr.brptr.data(), sizeof(long long) * (c->bcsr.nbrow + 1),
                  cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_brow, c->bcsr.brow.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_bcol, c->bcsr.bcol.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, st);
  if ((e = cudaMallocAsync(&d_count, sizeof(int) * (nb + 1), st))) return e;
  if ((e = cudaMallocAsync(&d_cursor, sizeof(int) * (nb + 1), st))) return e;
  cudaMemsetAsync(d_count, 0, sizeof(int) * (nb + 1), st);
  cudaMemsetAsync(d_cursor, 0, sizeof(int) * (nb + 1), st);
  if ((e = cudaMalloc(&c->d_bgptr, sizeof(int) * (nb + 1)))) return e;
  long long tot = (long long)c->nelem * kNab;
  unsigned g = (unsigned)((tot + 255) / 256);
  k_map_blocks<<<g, 256, 0, st>>>(c->nelem, c->d_lm, c->d_brptr, d_bcol, d_count, nullptr, nullptr,
                                  nullptr, 0, c->d_err);
  if ((e = scan_counts(d_count, c->d_bgptr, nb, st))) return e;
  int total = 0;
  cudaMemcpyAsync(&total, c->d_bgptr + nb, sizeof(int), cudaMemcpyDeviceToHost, st);
  if ((e = cudaStreamSynchronize(st))) return e;
  if ((e = cudaMalloc(&c->d_bglist, sizeof(int) * (size_t)(total > 0 ? total : 1)))) return e;
  k_map_blocks<<<g, 256, 0, st>>>(c->nelem, c->d_lm, c->d_brptr, d_bcol, nullptr, c->d_bgptr,
                                  d_cursor, c->d_bglist, 1, c->d_err);
  unsigned gb = (unsigned)((nb + 255) / 256);
  k_sort_lists<<<gb, 256, 0, st>>>(nb, c->d_bgptr, c->d_bglist, c->d_err);
  // PML elements and blocks
  std::vector<int> pml_elems, pml_local(c->nelem, -1);
  for (int i = 0; i < c->nelem; i++)
    if (c->h_cdomain[i] == 'A') {
      pml_local[i] = (int)pml_elems.size();
      pml_elems.push_back(i);
    }
  c->npml_elem = (int)pml_elems.size();
  if ((e = cudaMalloc(&c->d_pml_idx, sizeof(int) * nb))) return e;
  if (c->npml_elem > 0) {
    int *d_pml_local = nullptr, *d_isp = nullptr, *d_isp_scan = nullptr, *d_pcount_c = nullptr;
    if ((e = cudaMalloc(&c->d_pml_elems, sizeof(int) * c->npml_elem))) return e;
    cudaMemcpyAsync(c->d_pml_elems, pml_elems.data(), sizeof(int) * c->npml_elem,
                    cudaMemcpyHostToDevice, st);
    if ((e = cudaMallocAsync(&d_pml_local, sizeof(int) * c->nelem, st))) return e;
    cudaMemcpyAsync(d_pml_local, pml_local.data(), sizeof(int) * c->nelem, cudaMemcpyHostToDevice,
                    st);
    if ((e = cudaMallocAsync(&d_isp, sizeof(int) * (nb + 1), st))) return e;
    if ((e = cudaMallocAsync(&d_isp_scan, sizeof(int) * (nb + 1), st))) return e;
    cudaMemsetAsync(d_count, 0, sizeof(int) * (nb + 1), st);
    cudaMemsetAsync(d_isp, 0, sizeof(int) * (nb + 1), st);
    k_pml_count<<<gb, 256, 0, st>>>(nb, c->d_bgptr, c->d_bglist, c->d_cdomain, d_count, d_isp);
    if ((e = scan_counts(d_isp, d_isp_scan, nb, st))) return e;
    int npb = 0;
    cudaMemcpyAsync(&npb, d_isp_scan + nb, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st))) return e;
    c->npml_blocks = npb;
    if ((e = cudaMallocAsync(&d_pcount_c, sizeof(int) * (npb + 1), st))) return e;
    cudaMemsetAsync(d_pcount_c, 0, sizeof(int) * (npb + 1), st);
    k_compact_counts<<<gb, 256, 0, st>>>(nb, d_count, d_isp_scan, d_pcount_c);
    if ((e = cudaMalloc(&c->d_pgptr, sizeof(int) * (npb + 1)))) return e;
    if ((e = scan_counts(d_pcount_c, c->d_pgptr, npb, st))) return e;
    int ptot = 0;
    cudaMemcpyAsync(&ptot, c->d_pgptr + npb, sizeof(int), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st))) return e;
    if ((e = cudaMalloc(&c->d_pglist, sizeof(int) * (size_t)(ptot > 0 ? ptot : 1)))) return e;
    k_pml_fill<<<gb, 256, 0, st>>>(nb, c->d_bgptr, c->d_bglist, c->d_cdomain, d_isp_scan,
                                   d_pml_local, c->d_pgptr, c->d_pml_idx, c->d_pglist);
    if ((e = cudaMalloc(&c->d_pml_emat, sizeof(double2) * 9 * (size_t)c->npml_elem * kNab))) return e;
    cudaFreeAsync(d_pml_local, st);
    cudaFreeAsync(d_isp, st);
    cudaFreeAsync(d_isp_scan, st);
    cudaFreeAsync(d_pcount_c, st);
  } else {
    cudaMemsetAsync(c->d_pml_idx, 0xff, sizeof(int) * nb, st);
  }
  cudaFreeAsync(d_count, st);
  cudaFreeAsync(d_cursor, st);
  cudaFreeAsync(d_bcol, st);
  if ((e = cudaFuncSetAttribute(k_elem_basis, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)basis_smem())))
    return e;
  if ((e = cudaFuncSetAttribute(k_elem_pml, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)pml_smem())))
    return e;
  return cudaGetLastError();
}

cudaError_t build_basis(Ctx *c, cudaStream_t st) {
  cudaError_t e;
  const long long nb = c->bcsr.nblocks;
  if (!c->d_basis)
    if ((e = cudaMalloc(&c->d_basis, sizeof(double) * B_N * nb))) return e;
  double *d_eb = nullptr;
  if ((e = cudaMallocAsync(&d_eb, sizeof(double) * B_N * (size_t)c->nelem * kNab, st))) return e;
  k_elem_basis<<<c->nelem, kElemThreads, basis_smem(), st>>>(c->mv, c->dt, d_eb, c->d_err);
  k_gather_basis<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(nb, c->d_bgptr, c->d_bglist, d_eb,
                                                               c->d_basis);
  cudaFreeAsync(d_eb, st);
  if (!c->d_prim) {
    if ((e = cudaMalloc(&c->d_prim, sizeof(double) * (size_t)c->nzero))) return e;
    if ((e = cudaMalloc(&c->d_desc, sizeof(unsigned) * (size_t)c->nzero))) return e;
  }
  const long long g = ((long long)c->bcsr.nbrow * 32 + 255) / 256;
  k_build_prim<<<(unsigned)std::min<long long>(g, 1 << 20), 256, 0, st>>>(
      c->bcsr.nbrow, c->d_brptr, c->d_basis, nb, c->d_prim, c->d_desc);
  return cudaGetLastError();
}

cudaError_t build_pml_delta(Ctx *c, const PmlParams &pp, int slot, cudaStream_t st) {
  if (c->npml_elem == 0 || c->npml_blocks == 0) return cudaSuccess;
  double logr = std::log(pp.rcoeff);
  k_elem_pml<<<c->npml_elem, kElemThreads, pml_smem(), st>>>(c->mv, c->dt, c->d_pml_elems, pp, logr,
                                                            c->d_pml_emat, c->d_err);
  long long npb = c->npml_blocks;
  k_gather_pml<<<(unsigned)((npb + 255) / 256), 256, 0, st>>>(
      npb, c->d_pgptr, c->d_pglist, c->d_pml_emat, c->d_pml_delta + (size_t)slot * npb * 9);
  return cudaGetLastError();
}

template <int UNR>
static cudaError_t stream_range(Ctx *c, const SysTable &tab, int s0, int s1, double *ring_base,
                                long long slot_stride, int nslots, cudaStream_t st) {
  int nsm = 0, occ = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stream<UNR>, kStreamThreads, 0);
  if (occ < 1) occ = 1;
  const long long grid_need = (c->nzero + kStreamThreads - 1) / kStreamThreads;
  const unsigned grid = (unsigned)std::min<long long>((long long)nsm * occ, grid_need);
  k_stream<UNR><<<grid, kStreamThreads, 0, st>>>(c->nzero, c->d_prim, c->d_desc, c->d_basis,
                                                 c->bcsr.nblocks, c->d_pml_idx, c->d_pml_delta,
                                                 c->npml_blocks, tab, s0, s1, ring_base,
                                                 slot_stride, nslots);
  return cudaGetLastError();
}

static cudaError_t stream_pipe(Ctx *c, const SysTable &tab, int s0, int s1, double *ring_base,
                               long long slot_stride, int nslots, cudaStream_t st) {
  int nsm = 0, occ = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stream_pipe, kStreamThreads, 0);
  if (occ < 1) occ = 1;
  const long long grid_need = (c->nzero + kStreamThreads - 1) / kStreamThreads;
  const unsigned grid = (unsigned)std::min<long long>((long long)nsm * occ, grid_need);
  k_stream_pipe<<<grid, kStreamThreads, 0, st>>>(c->nzero, c->d_prim, c->d_desc, c->d_basis,
                                                 c->bcsr.nblocks, c->d_pml_idx, c->d_pml_delta,
                                                 c->npml_blocks, tab, s0, s1, ring_base,
                                                 slot_stride, nslots);
  return cudaGetLastError();
}

template <int T>
static cudaError_t stream_tma(Ctx *c, const SysTable &tab, int s0, int s1, double *ring_base,
                              long long slot_stride, int nslots, cudaStream_t st) {
  const size_t smem = sizeof(double2) * 2 * kMaxPass * T;
  cudaError_t e = cudaFuncSetAttribute(k_stream_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e) return e;
  int nsm = 0, occ = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stream_tma<T>, T, smem);
  if (occ < 1) occ = 1;
  const long long nchunk = (c->nzero + T - 1) / T;
  const unsigned grid = (unsigned)std::min<long long>((long long)nsm * occ, nchunk);
  k_stream_tma<T><<<grid, T, smem, st>>>(c->nzero, c->d_prim, c->d_desc, c->d_basis,
                                         c->bcsr.nblocks, c->d_pml_idx, c->d_pml_delta,
                                         c->npml_blocks, tab, s0, s1, ring_base, slot_stride,
                                         nslots);
  return cudaGetLastError();
}

template <int T, int NB>
static cudaError_t stream_ring(Ctx *c, const SysTable &tab, int s0, int s1, double *ring_base,
                               long long slot_stride, int nslots, cudaStream_t st) {
  const size_t smem = sizeof(double2) * NB * T;
  cudaError_t e = cudaFuncSetAttribute(k_stream_ring<T, NB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e) return e;
  int nsm = 0, occ = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stream_ring<T, NB>, T, smem);
  if (occ < 1) occ = 1;
  const long long nchunk = (c->nzero + T - 1) / T;
  const unsigned grid = (unsigned)std::min<long long>((long long)nsm * occ, nchunk);
  k_stream_ring<T, NB><<<grid, T, smem, st>>>(c->nzero, c->d_prim, c->d_desc, c->d_basis,
                                              c->bcsr.nblocks, c->d_pml_idx, c->d_pml_delta,
                                              c->npml_blocks, tab, s0, s1, ring_base, slot_stride,
                                              nslots);
  return cudaGetLastError();
}

template <int T, int NB>
static cudaError_t stream_big(Ctx *c, const SysParam *hsys, int s0, int s1, double *ring_base,
                              long long slot_stride, int nslots, cudaStream_t st) {
  SysTableBig tab;  // 24 KB; copied into the launch's parameters
  for (int k = 0; k < kMaxBatch; k++)
    tab.s[k] = k < s1 - s0 ? hsys[s0 + k] : SysParam{0.0, 0.0, 0, 0};
  const size_t smem = sizeof(double2) * NB * T;
  cudaError_t e = cudaFuncSetAttribute(k_stream_big<T, NB>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e) return e;
  int nsm = 0, occ = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_stream_big<T, NB>, T, smem);
  if (occ < 1) occ = 1;
  const long long nchunk = (c->nzero + T - 1) / T;
  const unsigned grid = (unsigned)std::min<long long>((long long)nsm * occ, nchunk);
  k_stream_big<T, NB><<<grid, T, smem, st>>>(c->nzero, c->d_prim, c->d_desc, c->d_basis,
                                             c->bcsr.nblocks, c->d_pml_idx, c->d_pml_delta,
                                             c->npml_blocks, tab, s0, s1, ring_base, slot_stride,
                                             nslots);
  return cudaGetLastError();
}

constexpr int kNumStreamVariants = 10;

// systems per launch of variant v: never more than the ring's slots, so every
// system of a launch lands in its own slot
static int variant_batch(int v, int nslots) {
  return std::min(v >= 8 ? kMaxBatch : kMaxPass, nslots);
}
static cudaError_t stream_variant(Ctx *c, int v, const SysParam *hsys, int s0, int s1,
                                  double *ring_base, long long slot_stride, int nslots,
                                  cudaStream_t st) {
  // the launch's systems travel as a kernel parameter, so a captured graph
  // keeps the values of its own call
  if (v == 8) return stream_big<512, 4>(c, hsys, s0, s1, ring_base, slot_stride, nslots, st);
  if (v == 9) return stream_big<256, 4>(c, hsys, s0, s1, ring_base, slot_stride, nslots, st);
  SysTable tab;
  for (int k = 0; k < kMaxPass; k++) tab.s[k] = k < s1 - s0 ? hsys[s0 + k] : SysParam{0.0, 0.0, 0, 0};
  switch (v) {
    case 0: return stream_range<1>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    case 1: return stream_range<2>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    case 2: return stream_range<4>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    case 3: return stream_pipe(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    case 4: return stream_tma<64>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    case 5: return stream_tma<128>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    case 6: return stream_ring<256, 4>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
    default: return stream_ring<512, 4>(c, tab, s0, s1, ring_base, slot_stride, nslots, st);
  }
}

// The first batch of a context times the streaming variants (1, 2 or 4
// entries per thread, software-pipelined, TMA bulk stores of all systems of a
// chunk, TMA staging ring of 256 or 512 entries with up to 16 systems per
// launch or, for larger rings, up to 1024) on its first launch of each -- each
// writes the same values
// -- compares the time per system and keeps the fastest for the life of the
// context.  A batch recorded into a CUDA graph before any tuning uses the
// 512-entry staging ring without timing.
cudaError_t launch_stream_batch(Ctx *c, int n, const SysParam *hsys, double *ring_base,
                                long long slot_stride, int nslots, cudaStream_t st) {
  cudaError_t e;
  int s0 = 0;
  if (c->stream_variant < 0) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    const char *env = std::getenv("FEM25_STREAM_VARIANT");
    if (env) {
      c->stream_variant = std::min(kNumStreamVariants - 1, std::max(0, std::atoi(env)));
    } else if (cs != cudaStreamCaptureStatusNone) {
      c->stream_variant = 7;
    } else {
      // every variant writes systems [0, its first launch), each in stream
      // order, so the slots end with the last system written
      cudaEvent_t ev[kNumStreamVariants + 1];
      for (auto &x : ev) cudaEventCreate(&x);
      cudaEventRecord(ev[0], st);
      for (int v = 0; v < kNumStreamVariants; v++) {
        const int s1 = std::min(n, variant_batch(v, nslots));
        if ((e = stream_variant(c, v, hsys, 0, s1, ring_base, slot_stride, nslots, st))) return e;
        cudaEventRecord(ev[v + 1], st);
      }
      cudaEventSynchronize(ev[kNumStreamVariants]);
      float best = 1e30f;
      for (int v = 0; v < kNumStreamVariants; v++) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[v], ev[v + 1]);
        t /= (float)std::min(n, variant_batch(v, nslots));
        if (t < best) {
          best = t;
          c->stream_variant = v;
        }
      }
      for (auto &x : ev) cudaEventDestroy(x);
      // the last tuning launch wrote the largest prefix; continue after it
      s0 = std::min(n, variant_batch(kNumStreamVariants - 1, nslots));
    }
  }
  const int per = std::min(n, variant_batch(c->stream_variant, nslots));
  for (; s0 < n; s0 += per) {
    const int s1 = std::min(n, s0 + per);
    if ((e = stream_variant(c, c->stream_variant, hsys, s0, s1, ring_base, slot_stride, nslots, st)))
      return e;
  }
  return cudaSuccess;
}

}  // namespace fem25
