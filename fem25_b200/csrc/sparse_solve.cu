// Sparse direct solve of one assembled system on the GPU: multifrontal LU
// with a nested-dissection ordering of the element mesh.  It stands in for
// the host MUMPS factor / solve hop of the reference (forward solve
// bielak25.f90:443-446, 545-551; transpose adjoint solve adjgrad.f90:327-341)
// on meshes far beyond the dense solve's reach, so the assemble -> solve ->
// misfit -> adjoint -> gradient loop stays on the device at the sizes of the
// benchmark meshes.
//
// Ordering (host, once per context).  The elements are bisected recursively
// along the longer side of their centroids' bounding box; the DOFs shared by
// the two halves that no coarser separator has taken form the separator of
// the tree node, and a leaf (at most kLeafElems elements) keeps every DOF of
// its elements that no separator took.  Because two DOFs are coupled only
// through an element they share, a separator splits the matrix graph.  The
// tree is the elimination tree: front t holds its own DOFs (the "fully
// summed" rows and columns, eliminated there) and its boundary: the DOFs of
// its subtree's elements owned by an ancestor, ordered by elimination.
//
// Factorisation (device), level by level from the leaves: every front of a
// level is assembled in a work buffer -- the CSR entries whose first
// eliminated DOF it owns, plus the update (Schur complement) blocks of its
// two children (extend-add) -- and partially factored: F11 = P L11 U11 with
// partial pivoting restricted to the fully summed rows, L21 = F21 U11^-1,
// U12 = L11^-1 P F12, update = F22 - L21 U12.  Fronts up to kSmallN rows are
// factored one CTA each in a single launch per level (blocked by panels of
// kNb columns factored in shared memory, rank-kNb trailing updates); larger
// fronts (the top levels of the tree) go to cuSOLVER getrf and cuBLAS trsm /
// gemm.  The factors (L11\U11 over L21, and U12) are copied to a store kept
// by the context; the update blocks live until the parent level has consumed
// them (two work buffers, alternating).
//
// Solve (device), one launch per level: forward elimination from the leaves,
// back substitution from the root, for op(A) = A, A^T (MUMPS ICNTL(9) != 1)
// or A^H; a CTA per (front, group of right-hand sides), the triangles solved
// in blocks of 32 rows.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cstdio>
#include <numeric>

#include "ctx.cuh"

namespace fem25 {

namespace sp {
constexpr int kLeafElems = 2;     // elements per leaf of the dissection
constexpr int kSmallN = 1024;     // fronts up to this many rows: one CTA each
constexpr int kNb = 8;            // panel width of the one-CTA factorisation
constexpr int kFacThreads = 256;  // threads of the one-CTA factorisation (128 measured slower)
constexpr int kThreads = 256;
constexpr int kRhsPerCta = 8;     // right-hand sides per solve CTA
constexpr int kLanes = 8;         // streams for the library-factored fronts of a level
}  // namespace sp

struct SpFront {
  int k, m;             // own (fully summed) and boundary DOFs
  int parent;           // -1: root
  int child[2];         // -1: none
  int level;            // depth in the dissection tree (root 0)
  long long own0;       // first own DOF in own[] (= elimination position)
  long long bnd0;       // first boundary DOF in bnd[]
  long long ea0;        // first entry of its extend-add map (ea[], m entries)
  long long fac0;       // factor store: L block [n][k] (ld n), then U12 [k][m] (ld k)
  long long work0;      // offset of its n x n front in its level's work buffer
};

// one stream of the library path with its own handles and workspace
struct SpLane {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  cusolverDnHandle_t sol = nullptr;
  cusolverDnParams_t par = nullptr;
  cublasHandle_t blas = nullptr;
  void *dwork = nullptr;
  size_t dwork_bytes = 0;
  std::vector<char> hwork;
  int *d_getrf_info = nullptr;
};

struct SparseLU {
  bool analysed = false, factored = false;
  int nfront = 0, nlevel = 0;
  std::vector<SpFront> fr;
  std::vector<std::vector<int>> lev;        // front ids per level, one-CTA fronts first
  std::vector<int> lev_nsmall, lev_nmax_small;  // per level: one-CTA fronts, their largest order
  std::vector<int> lev_kmax, lev_mmax;          // per level: largest own and boundary counts
  std::vector<long long> lev_work;          // work elements per level
  std::vector<long long> lev_ent0;          // first CSR-entry record of each level
  long long fac_elems = 0, max_work = 0;
  // device
  SpFront *d_fr = nullptr;
  int *d_own = nullptr, *d_bnd = nullptr, *d_ea = nullptr;
  int *d_lev_fronts = nullptr;              // all levels' front ids, concatenated
  std::vector<long long> lev_off;           // offset of each level in d_lev_fronts
  int *d_ent_idx = nullptr;                 // CSR entries by level, and their
  long long *d_ent_loc = nullptr;           // offsets in the level's work buffer
  double2 *d_fac = nullptr;                 // factor store
  int64_t *d_piv = nullptr;                 // pivots (1-based within each front), [NDOF]
  double2 *d_work[2] = {nullptr, nullptr};
  int *d_info = nullptr;                    // first zero pivot (front + 1), 0 = none
  SpLane lane[sp::kLanes];
  cudaEvent_t level_ready = nullptr;
};

// ---------------------------------------------------------------------------
// symbolic analysis (host)
// ---------------------------------------------------------------------------
namespace {

struct Builder {
  const int *lm_all;  // LM(3,25,NELEM), 1-based DOFs
  std::vector<double> cx, cz;
  std::vector<int> owner;    // DOF -> front (0-based DOF)
  std::vector<int> mark;     // scratch stamps per DOF
  int stamp = 0;
  std::vector<SpFront> fr;
  std::vector<std::vector<int>> own_list;   // per front, its own DOFs (ascending)
  std::vector<std::vector<int>> elems;      // per front, its subtree's elements

  int rec(std::vector<int> &E, int depth) {
    const int *lm = lm_all;
    if ((int)E.size() <= sp::kLeafElems) {
      std::vector<int> own;
      for (int e : E)
        for (int q = 0; q < kNee; q++) {
          const int d = lm[(size_t)e * kNee + q] - 1;
          if (d >= 0 && owner[d] == -1) {
            owner[d] = -3;  // claimed by this leaf (id given below)
            own.push_back(d);
          }
        }
      std::sort(own.begin(), own.end());
      const int id = (int)fr.size();
      for (int d : own) owner[d] = id;
      SpFront f{};
      f.k = (int)own.size();
      f.parent = -1;
      f.child[0] = f.child[1] = -1;
      f.level = depth;
      fr.push_back(f);
      own_list.push_back(std::move(own));
      elems.push_back(E);
      return id;
    }
    // bisect along the longer side of the centroids' bounding box
    double x0 = 1e300, x1 = -1e300, z0 = 1e300, z1 = -1e300;
    for (int e : E) {
      x0 = std::min(x0, cx[e]);
      x1 = std::max(x1, cx[e]);
      z0 = std::min(z0, cz[e]);
      z1 = std::max(z1, cz[e]);
    }
    const bool alongx = (x1 - x0) >= (z1 - z0);
    const size_t h = E.size() / 2;
    std::nth_element(E.begin(), E.begin() + h, E.end(), [&](int a, int b) {
      const double va = alongx ? cx[a] : cz[a], vb = alongx ? cx[b] : cz[b];
      return va < vb || (va == vb && a < b);
    });
    std::vector<int> E1(E.begin(), E.begin() + h), E2(E.begin() + h, E.end());
    // separator: free DOFs of both halves
    ++stamp;
    for (int e : E1)
      for (int q = 0; q < kNee; q++) {
        const int d = lm[(size_t)e * kNee + q] - 1;
        if (d >= 0) mark[d] = stamp;
      }
    std::vector<int> sep;
    for (int e : E2)
      for (int q = 0; q < kNee; q++) {
        const int d = lm[(size_t)e * kNee + q] - 1;
        if (d >= 0 && mark[d] == stamp && owner[d] == -1) {
          owner[d] = -2;  // taken by this separator (id given below)
          sep.push_back(d);
        }
      }
    const int c1 = rec(E1, depth + 1);
    const int c2 = rec(E2, depth + 1);
    std::sort(sep.begin(), sep.end());
    const int id = (int)fr.size();
    for (int d : sep) owner[d] = id;
    SpFront f{};
    f.k = (int)sep.size();
    f.parent = -1;
    f.child[0] = c1;
    f.child[1] = c2;
    f.level = depth;
    fr[c1].parent = id;
    fr[c2].parent = id;
    fr.push_back(f);
    own_list.push_back(std::move(sep));
    elems.push_back(E);
    return id;
  }
};

}  // namespace

// The dissection of a mesh (host only): the fronts with their own and
// boundary DOFs, elimination positions, levels and the offsets of every
// front's work and factor blocks.
struct FrontPlan {
  std::vector<SpFront> fr;
  std::vector<std::vector<int>> own, bnd;
  std::vector<long long> pos;
  std::vector<int> owner;
  std::vector<std::vector<int>> lev;
  std::vector<long long> lev_work;
  long long fac_elems = 0, bnd_tot = 0;
  int nlev = 0;
};

static int plan_fronts(int nelem, int n, const int *lm, const int *ieng, const double *xa,
                       const double *za, FrontPlan *pl, std::string *msg) {
  Builder b;
  b.lm_all = lm;
  b.cx.resize(nelem);
  b.cz.resize(nelem);
  for (int e = 0; e < nelem; e++) {
    double x = 0, z = 0;
    for (int a = 0; a < 4; a++) {
      const int p = ieng[4 * e + a] - 1;
      x += xa[p];
      z += za[p];
    }
    b.cx[e] = 0.25 * x;
    b.cz[e] = 0.25 * z;
  }
  b.owner.assign(n, -1);
  b.mark.assign(n, 0);
  std::vector<int> E(nelem);
  std::iota(E.begin(), E.end(), 0);
  b.rec(E, 0);
  for (int d = 0; d < n; d++)
    if (b.owner[d] < 0) {
      *msg = "sparse solve: a DOF belongs to no element";
      return FEM25_ERR_PATTERN;
    }
  const int nf = (int)b.fr.size();
  // elimination positions (postorder = front id order)
  std::vector<long long> &pos = pl->pos;
  pos.assign(n, 0);
  long long p = 0;
  for (int t = 0; t < nf; t++) {
    b.fr[t].own0 = p;
    for (int d : b.own_list[t]) pos[d] = p++;
  }
  // boundaries: DOFs of the subtree's elements owned by an ancestor (id > t)
  std::vector<std::vector<int>> &bnd = pl->bnd;
  bnd.assign(nf, {});
  {
    std::vector<int> seen(n, -1);
    for (int t = 0; t < nf; t++) {
      std::vector<int> &B = bnd[t];
      for (int e : b.elems[t])
        for (int q = 0; q < kNee; q++) {
          const int d = lm[(size_t)e * kNee + q] - 1;
          if (d >= 0 && b.owner[d] > t && seen[d] != t) {
            seen[d] = t;
            B.push_back(d);
          }
        }
      std::sort(B.begin(), B.end(), [&](int x, int y) { return pos[x] < pos[y]; });
      b.fr[t].m = (int)B.size();
      b.elems[t].clear();
      b.elems[t].shrink_to_fit();
    }
  }
  // levels, offsets
  int nlev = 0;
  for (auto &f : b.fr) nlev = std::max(nlev, f.level + 1);
  pl->lev.assign(nlev, {});
  pl->lev_work.assign(nlev, 0);
  long long bnd_tot = 0, fac = 0;
  for (int t = 0; t < nf; t++) {
    SpFront &f = b.fr[t];
    const long long nn = (long long)f.k + f.m;
    f.bnd0 = bnd_tot;
    f.ea0 = bnd_tot;
    bnd_tot += f.m;
    f.fac0 = fac;
    fac += nn * f.k + (long long)f.k * f.m;
    f.work0 = pl->lev_work[f.level];
    pl->lev_work[f.level] += nn * nn;
    pl->lev[f.level].push_back(t);
  }
  pl->fac_elems = fac;
  pl->bnd_tot = bnd_tot;
  pl->nlev = nlev;
  pl->fr = std::move(b.fr);
  pl->own = std::move(b.own_list);
  pl->owner = std::move(b.owner);
  return 0;
}

// fronts, levels, factor bytes, largest level work bytes, largest own count,
// largest front order, real flops of one factorisation (8 per complex
// multiply-add)
static void plan_stats(const std::vector<SpFront> &fr, long long fac_elems,
                       const std::vector<long long> &lev_work, long long *out) {
  int kmax = 0, nmax = 0, nlev = 0;
  double flops = 0.0;
  for (const SpFront &f : fr) {
    kmax = std::max(kmax, f.k);
    nmax = std::max(nmax, f.k + f.m);
    nlev = std::max(nlev, f.level + 1);
    const double k = f.k, m = f.m;
    flops += 8.0 / 3.0 * k * k * k + 8.0 * k * k * m + 8.0 * k * m * m;
  }
  long long wmax = 0;
  for (long long w : lev_work) wmax = std::max(wmax, w);
  out[0] = (long long)fr.size();
  out[1] = nlev;
  out[2] = fac_elems * 16;
  out[3] = wmax * 16;
  out[4] = kmax;
  out[5] = nmax;
  out[6] = (long long)flops;
}

int sparse_plan_info(int nelem, int ndof, const int *lm, const int *ieng, const double *x,
                     const double *z, long long *out, std::string *msg) {
  FrontPlan pl;
  const int r = plan_fronts(nelem, ndof, lm, ieng, x, z, &pl, msg);
  if (r) return r;
  plan_stats(pl.fr, pl.fac_elems, pl.lev_work, out);
  return 0;
}

// Builds the ordering, the fronts, the extend-add maps and the CSR-entry map;
// uploads them.  0, or a FEM25 status with *msg.
static int sparse_analyse(Ctx *c, SparseLU *s, cudaStream_t st, std::string *msg) {
  const int n = c->ndof;
  FrontPlan pl;
  {
    const int r = plan_fronts(c->nelem, n, c->h_lm.data(), c->h_ieng.data(), c->h_x.data(),
                              c->h_z.data(), &pl, msg);
    if (r) return r;
  }
  const int nf = (int)pl.fr.size();
  const int nlev = pl.nlev;
  const std::vector<long long> &pos = pl.pos;
  const std::vector<std::vector<int>> &bnd = pl.bnd;
  struct {
    std::vector<SpFront> &fr;
    std::vector<std::vector<int>> &own_list;
    std::vector<int> &owner;
  } b{pl.fr, pl.own, pl.owner};
  // index of DOF d in front t (own: by position; boundary: by search)
  auto local = [&](int t, int d) -> int {
    const SpFront &f = b.fr[t];
    if (b.owner[d] == t) return (int)(pos[d] - f.own0);
    const std::vector<int> &B = bnd[t];
    auto it = std::lower_bound(B.begin(), B.end(), d,
                               [&](int x, int y) { return pos[x] < pos[y]; });
    if (it == B.end() || *it != d) return -1;
    return f.k + (int)(it - B.begin());
  };
  s->lev = pl.lev;
  s->lev_work = pl.lev_work;
  s->fac_elems = pl.fac_elems;
  s->max_work = 0;
  for (long long w : s->lev_work) s->max_work = std::max(s->max_work, w);
  const long long bnd_tot = pl.bnd_tot;
  // extend-add maps: child boundary DOF -> index in the parent's front
  std::vector<int> ea(bnd_tot), own_all(n), bnd_all(bnd_tot);
  for (int t = 0; t < nf; t++) {
    const SpFront &f = b.fr[t];
    std::copy(b.own_list[t].begin(), b.own_list[t].end(), own_all.begin() + f.own0);
    std::copy(bnd[t].begin(), bnd[t].end(), bnd_all.begin() + f.bnd0);
    for (int i = 0; i < f.m; i++) {
      const int li = f.parent >= 0 ? local(f.parent, bnd[t][i]) : -1;
      if (li < 0) {
        *msg = "sparse solve: a boundary DOF is missing from the parent front";
        return FEM25_ERR_PATTERN;
      }
      ea[f.ea0 + i] = li;
    }
  }
  // CSR entries -> (front, local offset), grouped by level
  std::vector<int> jc(c->nzero);
  cudaError_t e;
  if ((e = cudaMemcpy(jc.data(), c->d_jcptr, sizeof(int) * c->nzero, cudaMemcpyDeviceToHost))) {
    *msg = std::string("sparse solve: ") + cudaGetErrorString(e);
    return FEM25_ERR_CUDA;
  }
  // two passes over the rows in chunks: count the entries of each level per
  // chunk, then place each entry at its level's and chunk's next slot
  const int nchunk = 256;
  const int rows_per = (n + nchunk - 1) / nchunk;
  std::vector<long long> cnt((size_t)nchunk * nlev, 0);
  int bad = 0;
  auto entry_front = [&](int i, int j) { return pos[i] <= pos[j] ? b.owner[i] : b.owner[j]; };
#pragma omp parallel for schedule(dynamic, 1)
  for (int ch = 0; ch < nchunk; ch++) {
    long long *cc = cnt.data() + (size_t)ch * nlev;
    const int i1 = std::min(n, (ch + 1) * rows_per);
    for (int i = ch * rows_per; i < i1; i++)
      for (int q = c->h_irptr[i] - 1; q < c->h_irptr[i + 1] - 1; q++)
        cc[b.fr[entry_front(i, jc[q] - 1)].level]++;
  }
  s->lev_ent0.assign(nlev + 1, 0);
  std::vector<long long> cur((size_t)nchunk * nlev);
  {
    long long acc = 0;
    for (int l = 0; l < nlev; l++) {
      s->lev_ent0[l] = acc;
      for (int ch = 0; ch < nchunk; ch++) {
        cur[(size_t)ch * nlev + l] = acc;
        acc += cnt[(size_t)ch * nlev + l];
      }
    }
    s->lev_ent0[nlev] = acc;
  }
  std::vector<int> sidx(c->nzero);
  std::vector<long long> sloc(c->nzero);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : bad)
  for (int ch = 0; ch < nchunk; ch++) {
    long long *cc = cur.data() + (size_t)ch * nlev;
    const int i1 = std::min(n, (ch + 1) * rows_per);
    for (int i = ch * rows_per; i < i1; i++)
      for (int q = c->h_irptr[i] - 1; q < c->h_irptr[i + 1] - 1; q++) {
        const int j = jc[q] - 1;
        const int t = entry_front(i, j);
        const int li = local(t, i), lj = local(t, j);
        if (li < 0 || lj < 0) {
          bad++;
          continue;
        }
        const long long nn = (long long)b.fr[t].k + b.fr[t].m;
        const long long o = cc[b.fr[t].level]++;
        sidx[o] = q;
        sloc[o] = b.fr[t].work0 + li + (long long)lj * nn;
      }
  }
  if (bad) {
    *msg = "sparse solve: a matrix entry couples DOFs of no common front";
    return FEM25_ERR_PATTERN;
  }
  std::vector<int>().swap(jc);
  // one-CTA fronts first in each level's list
  s->lev_nsmall.assign(nlev, 0);
  s->lev_nmax_small.assign(nlev, 0);
  s->lev_kmax.assign(nlev, 0);
  s->lev_mmax.assign(nlev, 0);
  for (int t = 0; t < nf; t++) {
    s->lev_kmax[b.fr[t].level] = std::max(s->lev_kmax[b.fr[t].level], b.fr[t].k);
    s->lev_mmax[b.fr[t].level] = std::max(s->lev_mmax[b.fr[t].level], b.fr[t].m);
  }
  for (int l = 0; l < nlev; l++) {
    std::stable_partition(s->lev[l].begin(), s->lev[l].end(), [&](int t) {
      return b.fr[t].k + b.fr[t].m <= sp::kSmallN;
    });
    for (int t : s->lev[l])
      if (b.fr[t].k + b.fr[t].m <= sp::kSmallN) {
        s->lev_nsmall[l]++;
        s->lev_nmax_small[l] = std::max(s->lev_nmax_small[l], b.fr[t].k + b.fr[t].m);
      }
  }
  // level front lists, concatenated
  std::vector<int> lf;
  s->lev_off.assign(nlev + 1, 0);
  for (int l = 0; l < nlev; l++) {
    s->lev_off[l] = (long long)lf.size();
    lf.insert(lf.end(), s->lev[l].begin(), s->lev[l].end());
  }
  s->lev_off[nlev] = (long long)lf.size();
  // upload
  auto up = [&](void **d, const void *h, size_t bytes) -> cudaError_t {
    cudaError_t r = cudaMalloc(d, bytes ? bytes : 16);
    if (r == cudaSuccess && bytes) r = cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice);
    return r;
  };
  if ((e = up((void **)&s->d_fr, b.fr.data(), sizeof(SpFront) * nf)) ||
      (e = up((void **)&s->d_own, own_all.data(), sizeof(int) * n)) ||
      (e = up((void **)&s->d_bnd, bnd_all.data(), sizeof(int) * bnd_tot)) ||
      (e = up((void **)&s->d_ea, ea.data(), sizeof(int) * bnd_tot)) ||
      (e = up((void **)&s->d_lev_fronts, lf.data(), sizeof(int) * lf.size())) ||
      (e = up((void **)&s->d_ent_idx, sidx.data(), sizeof(int) * sidx.size())) ||
      (e = up((void **)&s->d_ent_loc, sloc.data(), sizeof(long long) * sloc.size()))) {
    *msg = std::string("sparse solve: ") + cudaGetErrorString(e) + " (symbolic tables)";
    return FEM25_ERR_ALLOC;
  }
  s->fr = std::move(b.fr);
  s->nfront = nf;
  s->nlevel = nlev;
  s->analysed = true;
  (void)st;
  return 0;
}

// ---------------------------------------------------------------------------
// numeric factorisation (device)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfms(double2 acc, double2 a, double2 b) {  // acc - a b
  return make_double2(acc.x - a.x * b.x + a.y * b.y, acc.y - a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// CSR entries of one level into their fronts' work buffers
__global__ void k_sp_assemble(long long n, const int *__restrict__ idx,
                              const long long *__restrict__ loc, const double2 *__restrict__ csr,
                              double2 *__restrict__ work) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    work[loc[i]] = csr[idx[i]];
}

// extend-add of child slot `slot` of every front of the level: one CTA per front
__global__ void k_sp_extend_add(const int *__restrict__ fronts, const SpFront *__restrict__ fr,
                                const int *__restrict__ ea, const double2 *__restrict__ wchild,
                                double2 *__restrict__ work, int slot) {
  const SpFront f = fr[fronts[blockIdx.x]];
  const int ch = f.child[slot];
  if (ch < 0) return;
  const SpFront g = fr[ch];
  const long long nf = (long long)f.k + f.m, ng = (long long)g.k + g.m;
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = blockIdx.y * nw + (threadIdx.x >> 5); j < g.m; j += gridDim.y * nw) {
    const double2 *src = wchild + g.work0 + g.k + (long long)(g.k + j) * ng;
    double2 *dst = work + f.work0 + (long long)ea[g.ea0 + j] * nf;
    for (int i = lane; i < g.m; i += 32) {
      const double2 v = src[i];
      double2 *o = dst + ea[g.ea0 + i];
      o->x += v.x;
      o->y += v.y;
    }
  }
}

// Partial LU of one front per CTA, blocked by panels of kNb columns: the
// panel (rows jb..n-1) is factored in shared memory with partial pivoting
// restricted to the fully summed rows, its row interchanges are applied to
// the front's other columns, the panel's U block (rows jb..jb+nb-1) is
// solved with the panel's unit lower triangle, and the trailing block is
// updated by a rank-nb product: a warp per pair of columns, their U values
// in registers, the panel rows read from shared memory.  In place in the
// work buffer; pivots 1-based within the front.
__global__ void __launch_bounds__(sp::kFacThreads) k_sp_factor_blk(
    const int *__restrict__ fronts, int nfr, const SpFront *__restrict__ fr,
    double2 *__restrict__ work, int64_t *__restrict__ piv, int *__restrict__ info) {
  extern __shared__ double2 P[];  // panel: P[r + c * pr], r < pr = n - jb, c < nb
  __shared__ double red_v[sp::kFacThreads / 32];
  __shared__ int red_i[sp::kFacThreads / 32];
  __shared__ int swp[sp::kNb];
  const int b = blockIdx.x;
  if (b >= nfr) return;
  const int t = fronts[b];
  const SpFront f = fr[t];
  const int k = f.k, n = f.k + f.m;
  double2 *F = work + f.work0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = (int)(blockDim.x >> 5);
  for (int jb = 0; jb < k; jb += sp::kNb) {
    const int nb = min(sp::kNb, k - jb), pr = n - jb, kr = k - jb;
    // 1. the panel to shared memory
    for (int c = 0; c < nb; c++)
      for (int r = tid; r < pr; r += blockDim.x) P[r + c * pr] = F[jb + r + (long long)(jb + c) * n];
    __syncthreads();
    // 2. unblocked LU of the panel; pivots among its first kr rows
    for (int j = 0; j < nb; j++) {
      double best = -1.0;
      int bi = j;
      for (int r = j + tid; r < kr; r += blockDim.x) {
        const double2 v = P[r + j * pr];
        const double a = fabs(v.x) + fabs(v.y);
        if (a > best) {
          best = a;
          bi = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        red_v[warp] = best;
        red_i[warp] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double bb = -1.0;
        int ii = j;
        for (int w = 0; w < nw; w++)
          if (red_v[w] > bb || (red_v[w] == bb && red_i[w] < ii)) {
            bb = red_v[w];
            ii = red_i[w];
          }
        swp[j] = ii;
        piv[f.own0 + jb + j] = jb + ii + 1;
        if (bb <= 0.0) atomicCAS(info, 0, t + 1);
      }
      __syncthreads();
      const int pj = swp[j];
      if (pj != j)
        for (int c = tid; c < nb; c += blockDim.x) {
          const double2 x = P[j + c * pr];
          P[j + c * pr] = P[pj + c * pr];
          P[pj + c * pr] = x;
        }
      __syncthreads();
      const double2 d = P[j + j * pr];
      const bool zero = d.x == 0.0 && d.y == 0.0;
      for (int r = j + 1 + tid; r < pr; r += blockDim.x)
        P[r + j * pr] = zero ? make_double2(0.0, 0.0) : cdiv(P[r + j * pr], d);
      __syncthreads();
      for (int c = j + 1; c < nb; c++) {
        const double2 u = P[j + c * pr];
        for (int r = j + 1 + tid; r < pr; r += blockDim.x)
          P[r + c * pr] = cfms(P[r + c * pr], P[r + j * pr], u);
      }
      __syncthreads();
    }
    // 3. the panel back; 4. its interchanges on the other columns
    for (int c = 0; c < nb; c++)
      for (int r = tid; r < pr; r += blockDim.x) F[jb + r + (long long)(jb + c) * n] = P[r + c * pr];
    for (int c = tid; c < n - nb; c += blockDim.x) {
      double2 *col = F + (long long)(c < jb ? c : c + nb) * n + jb;
      for (int j = 0; j < nb; j++) {
        const int pj = swp[j];
        if (pj != j) {
          const double2 x = col[j];
          col[j] = col[pj];
          col[pj] = x;
        }
      }
    }
    __syncthreads();
    // 5. the U block: unit lower solve with the panel's top nb x nb triangle
    for (int cc = jb + nb + tid; cc < n; cc += blockDim.x) {
      double2 *col = F + (long long)cc * n + jb;
      double2 x[sp::kNb];
#pragma unroll
      for (int i = 0; i < sp::kNb; i++) x[i] = i < nb ? col[i] : make_double2(0.0, 0.0);
#pragma unroll
      for (int i = 1; i < sp::kNb; i++)
#pragma unroll
        for (int j = 0; j < i; j++) x[i] = cfms(x[i], P[i + j * pr], x[j]);
#pragma unroll
      for (int i = 0; i < sp::kNb; i++)
        if (i < nb) col[i] = x[i];
    }
    __syncthreads();
    // 6. trailing update, rows and columns from jb + nb: a warp per pair of
    // columns (each panel value read from shared memory feeds two columns)
    const int c0 = jb + nb;
    for (int cp = c0 + 2 * warp; cp < n; cp += 2 * nw) {
      const bool two = cp + 1 < n;
      double2 u0[sp::kNb], u1[sp::kNb];
#pragma unroll
      for (int j = 0; j < sp::kNb; j++) {
        u0[j] = j < nb ? F[jb + j + (long long)cp * n] : make_double2(0.0, 0.0);
        u1[j] = (two && j < nb) ? F[jb + j + (long long)(cp + 1) * n] : make_double2(0.0, 0.0);
      }
      double2 *col0 = F + (long long)cp * n, *col1 = col0 + n;
      for (int r = c0 + lane; r < n; r += 32) {
        double2 a0 = col0[r], a1 = two ? col1[r] : make_double2(0.0, 0.0);
        const double2 *pl = P + (r - jb);
#pragma unroll
        for (int j = 0; j < sp::kNb; j++) {
          const double2 l = j < nb ? pl[j * pr] : make_double2(0.0, 0.0);
          a0 = cfms(a0, l, u0[j]);
          a1 = cfms(a1, l, u1[j]);
        }
        col0[r] = a0;
        if (two) col1[r] = a1;
      }
    }
    __syncthreads();
  }
}

// a library-factored front's zero pivot into the status word
__global__ void k_sp_getrf_status(const int *getrf_info, int *info, int front) {
  if (*getrf_info > 0) atomicCAS(info, 0, front + 1);
}

// row interchanges of a front's pivots on columns [c0, c1) (laswp)
__global__ void k_sp_laswp(double2 *F, int n, int k, int c0, int c1, const int64_t *piv) {
  for (int cidx = c0 + blockIdx.x * blockDim.x + threadIdx.x; cidx < c1;
       cidx += gridDim.x * blockDim.x)
    for (int j = 0; j < k; j++) {
      const int p = (int)piv[j] - 1;
      if (p != j) {
        double2 *a = F + j + (long long)cidx * n, *b = F + p + (long long)cidx * n;
        const double2 x = *a;
        *a = *b;
        *b = x;
      }
    }
}

// factors of the level's fronts to the store: the first k columns (L11\U11
// over L21, n x k) and U12 (rows 0..k-1 of columns k..n-1, k x m, ld k)
__global__ void k_sp_store(const int *__restrict__ fronts, const SpFront *__restrict__ fr,
                           const double2 *__restrict__ work, double2 *__restrict__ fac) {
  const SpFront f = fr[fronts[blockIdx.x]];
  const long long n = (long long)f.k + f.m;
  const double2 *F = work + f.work0;
  double2 *L = fac + f.fac0, *U = L + n * f.k;
  const long long stride = (long long)gridDim.y * blockDim.x;
  for (long long q = blockIdx.y * blockDim.x + threadIdx.x; q < n * f.k; q += stride) L[q] = F[q];
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = blockIdx.y * nw + (threadIdx.x >> 5); j < f.m; j += gridDim.y * nw)
    for (int i = lane; i < f.k; i += 32) U[i + (long long)j * f.k] = F[i + (f.k + j) * n];
}

// ---------------------------------------------------------------------------
// solve (device): x is [nrhs][NDOF]
// ---------------------------------------------------------------------------
// The triangular solves of one front, blocked by 32 rows: warp 0 solves the
// 32 x 32 diagonal triangle of a block with the block's right-hand-side
// values in registers (lane = row; values passed on by shuffles), the CTA
// then updates the rows still to come with the solved block (kept in shared
// memory): two CTA barriers per 32 rows.  Row r of the own block is the DOF
// own[r]; the right-hand sides [r0, r0 + nr) of x (one CTA per group of
// kRhsPerCta).
//   op(A) = A    forward: interchanges, L11 (unit lower), x_b -= L21 x_own
//                backward: x_own -= U12 x_b, U11 (upper)
//   A^T / A^H    forward: U11^op (lower), x_b -= U12^op x_own
//                backward: x_own -= L21^op x_b, L11^op (unit upper), inverse
//                interchanges
// The boundary rows x_b of a front belong to ancestors; fronts of one level
// may share them, so the forward updates add with atomics.
struct SolveArgs {
  const int *fronts;
  const SpFront *fr;
  const int *own, *bnd;
  const double2 *fac;
  const int64_t *piv;
  double2 *x;
  int ndof, nrhs, trans;  // trans 0: A, 1: A^T, 2: A^H
};

__device__ __forceinline__ double2 sp_op(double2 v, int trans) {
  return trans == 2 ? cconj(v) : v;
}

// element (i, j) of op(T) for the front's F11 (ld n) or L21 rows: op(T)(i, j)
// = T(i, j) for A, T(j, i) (conjugated for A^H) for A^T / A^H
__device__ __forceinline__ double2 sp_el(const double2 *T, long long n, int i, int j, int trans) {
  return trans == 0 ? T[i + (long long)j * n] : sp_op(T[j + (long long)i * n], trans);
}

template <int R>
__global__ void __launch_bounds__(sp::kThreads) k_sp_solve_fwd(SolveArgs a) {
  __shared__ double2 xs[32][R];
  __shared__ double2 tb[32][33];  // the block's diagonal triangle, op applied
  const SpFront f = a.fr[a.fronts[blockIdx.x]];
  const int r0 = blockIdx.y * R, nr = min(R, a.nrhs - r0);
  if (nr <= 0 || f.k == 0) return;
  const long long n = (long long)f.k + f.m;
  const int k = f.k, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int *ow = a.own + f.own0;
  const double2 *F = a.fac + f.fac0;          // F11 and L21, ld n
  double2 *x = a.x + (long long)r0 * a.ndof;
  const int tr = a.trans;
  if (tr == 0 && tid < nr) {  // row interchanges of P
    double2 *xr = x + (long long)tid * a.ndof;
    for (int j = 0; j < k; j++) {
      const int p = (int)a.piv[f.own0 + j] - 1;
      if (p != j) {
        const double2 t = xr[ow[j]];
        xr[ow[j]] = xr[ow[p]];
        xr[ow[p]] = t;
      }
    }
  }
  __syncthreads();
  // lower triangle T: L11 (unit) for A, U11^op (non-unit) for A^T / A^H
  for (int jb = 0; jb < k; jb += 32) {
    const int nb = min(32, k - jb);
    for (int q = tid; q < nb * nb; q += blockDim.x) {
      const int i = q % nb, j = q / nb;
      if (i > j) tb[i][j] = sp_el(F, n, jb + i, jb + j, tr);
      if (i == j && tr != 0) tb[i][i] = cdiv(make_double2(1.0, 0.0), sp_el(F, n, jb + i, jb + i, tr));
    }
    __syncthreads();
    if (warp == 0) {
      double2 v[R];
#pragma unroll
      for (int s = 0; s < R; s++)
        v[s] = (lane < nb && s < nr) ? x[(long long)s * a.ndof + ow[jb + lane]] : make_double2(0.0, 0.0);
      for (int i = 0; i < nb; i++) {
        if (tr != 0 && lane == i) {
          const double2 d = tb[i][i];  // reciprocal of the diagonal
#pragma unroll
          for (int s = 0; s < R; s++) v[s] = cmul(v[s], d);
        }
        const double2 tli = (lane > i && lane < nb) ? tb[lane][i] : make_double2(0.0, 0.0);
#pragma unroll
        for (int s = 0; s < R; s++) {
          const double2 xi = make_double2(__shfl_sync(0xffffffffu, v[s].x, i),
                                          __shfl_sync(0xffffffffu, v[s].y, i));
          if (lane > i && lane < nb) v[s] = cfms(v[s], tli, xi);
        }
      }
      if (lane < nb)
#pragma unroll
        for (int s = 0; s < R; s++)
          if (s < nr) {
            x[(long long)s * a.ndof + ow[jb + lane]] = v[s];
            xs[lane][s] = v[s];
          }
    }
    __syncthreads();
    for (int r = jb + nb + tid; r < k; r += blockDim.x) {
      double2 acc[R];
#pragma unroll
      for (int s = 0; s < R; s++)
        acc[s] = s < nr ? x[(long long)s * a.ndof + ow[r]] : make_double2(0.0, 0.0);
      for (int i = 0; i < nb; i++) {
        const double2 t = sp_el(F, n, r, jb + i, tr);
#pragma unroll
        for (int s = 0; s < R; s++) acc[s] = cfms(acc[s], t, xs[i][s]);
      }
#pragma unroll
      for (int s = 0; s < R; s++)
        if (s < nr) x[(long long)s * a.ndof + ow[r]] = acc[s];
    }
    __syncthreads();
  }
}

// The rectangular part of a front's solve step, spread over CTAs of
// kThreads rows each (blockIdx.y: row tile, blockIdx.z: group of
// right-hand sides):
//   fwd: boundary rows   x_b -= L21 x_own (A), U12^op x_own (A^T / A^H),
//        added with atomics (fronts of a level share boundary rows)
//   bwd: own rows        x_own -= U12 x_b (A), L21^op x_b (A^T / A^H)
// The right-hand-side values of the summed index pass through shared memory
// in chunks of kThreads, so each thread's dot product streams its matrix row.
template <int R>
__global__ void __launch_bounds__(sp::kThreads) k_sp_solve_rect(SolveArgs a, int fwd) {
  __shared__ double2 xc[sp::kThreads][R];
  const SpFront f = a.fr[a.fronts[blockIdx.x]];
  const int r0 = blockIdx.z * R, nr = min(R, a.nrhs - r0);
  const int rows = fwd ? f.m : f.k, cols = fwd ? f.k : f.m;
  const int row0 = blockIdx.y * blockDim.x;
  if (nr <= 0 || row0 >= rows || cols == 0) return;
  const long long n = (long long)f.k + f.m;
  const int k = f.k, tid = threadIdx.x, tr = a.trans;
  const double2 *F = a.fac + f.fac0, *U12 = F + n * k;
  const int *rowidx = (fwd ? a.bnd + f.bnd0 : a.own + f.own0);
  const int *colidx = (fwd ? a.own + f.own0 : a.bnd + f.bnd0);
  double2 *x = a.x + (long long)r0 * a.ndof;
  const int r = row0 + tid;
  double2 acc[R];
#pragma unroll
  for (int s = 0; s < R; s++) acc[s] = make_double2(0.0, 0.0);
  for (int c0 = 0; c0 < cols; c0 += blockDim.x) {
    const int nc = min((int)blockDim.x, cols - c0);
    __syncthreads();
    if (tid < nc) {
      const int d = colidx[c0 + tid];
#pragma unroll
      for (int s = 0; s < R; s++)
        xc[tid][s] = s < nr ? x[(long long)s * a.ndof + d] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    if (r < rows) {
#pragma unroll 4
      for (int j = 0; j < nc; j++) {
        const int c = c0 + j;
        // element (r, c) of the rectangular block
        double2 t;
        if (fwd)
          t = tr == 0 ? F[k + r + (long long)c * n] : sp_op(U12[c + (long long)r * k], tr);
        else
          t = tr == 0 ? U12[r + (long long)c * k] : sp_op(F[k + c + (long long)r * n], tr);
#pragma unroll
        for (int s = 0; s < R; s++) acc[s] = cfms(acc[s], t, xc[j][s]);
      }
    }
  }
  if (r >= rows) return;
  const int d = rowidx[r];
#pragma unroll
  for (int s = 0; s < R; s++)
    if (s < nr) {
      double2 *o = x + (long long)s * a.ndof + d;
      if (fwd) {  // acc = -(product)
        atomicAdd(reinterpret_cast<double *>(o), acc[s].x);
        atomicAdd(reinterpret_cast<double *>(o) + 1, acc[s].y);
      } else {
        *o = make_double2(o->x + acc[s].x, o->y + acc[s].y);
      }
    }
}

template <int R>
__global__ void __launch_bounds__(sp::kThreads) k_sp_solve_bwd(SolveArgs a) {
  __shared__ double2 xs[32][R];
  __shared__ double2 tb[32][33];  // the block's diagonal triangle, op applied
  const SpFront f = a.fr[a.fronts[blockIdx.x]];
  const int r0 = blockIdx.y * R, nr = min(R, a.nrhs - r0);
  if (nr <= 0 || f.k == 0) return;
  const long long n = (long long)f.k + f.m;
  const int k = f.k, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int *ow = a.own + f.own0;
  const double2 *F = a.fac + f.fac0;
  double2 *x = a.x + (long long)r0 * a.ndof;
  const int tr = a.trans;
  // upper triangle T: U11 (non-unit) for A, L11^op (unit) for A^T / A^H;
  // blocks of 32 rows from the bottom
  for (int jb = ((k - 1) / 32) * 32; jb >= 0; jb -= 32) {
    const int nb = min(32, k - jb);
    for (int q = tid; q < nb * nb; q += blockDim.x) {
      const int i = q % nb, j = q / nb;
      if (i < j) tb[i][j] = sp_el(F, n, jb + i, jb + j, tr);
      if (i == j && tr == 0) tb[i][i] = cdiv(make_double2(1.0, 0.0), sp_el(F, n, jb + i, jb + i, tr));
    }
    __syncthreads();
    if (warp == 0) {
      double2 v[R];
#pragma unroll
      for (int s = 0; s < R; s++)
        v[s] = (lane < nb && s < nr) ? x[(long long)s * a.ndof + ow[jb + lane]] : make_double2(0.0, 0.0);
      for (int i = nb - 1; i >= 0; i--) {
        if (tr == 0 && lane == i) {
          const double2 d = tb[i][i];  // reciprocal of the diagonal
#pragma unroll
          for (int s = 0; s < R; s++) v[s] = cmul(v[s], d);
        }
        const double2 tli = lane < i ? tb[lane][i] : make_double2(0.0, 0.0);
#pragma unroll
        for (int s = 0; s < R; s++) {
          const double2 xi = make_double2(__shfl_sync(0xffffffffu, v[s].x, i),
                                          __shfl_sync(0xffffffffu, v[s].y, i));
          if (lane < i) v[s] = cfms(v[s], tli, xi);
        }
      }
      if (lane < nb)
#pragma unroll
        for (int s = 0; s < R; s++)
          if (s < nr) {
            x[(long long)s * a.ndof + ow[jb + lane]] = v[s];
            xs[lane][s] = v[s];
          }
    }
    __syncthreads();
    for (int r = tid; r < jb; r += blockDim.x) {
      double2 acc[R];
#pragma unroll
      for (int s = 0; s < R; s++)
        acc[s] = s < nr ? x[(long long)s * a.ndof + ow[r]] : make_double2(0.0, 0.0);
      for (int i = 0; i < nb; i++) {
        const double2 t = sp_el(F, n, r, jb + i, tr);
#pragma unroll
        for (int s = 0; s < R; s++) acc[s] = cfms(acc[s], t, xs[i][s]);
      }
#pragma unroll
      for (int s = 0; s < R; s++)
        if (s < nr) x[(long long)s * a.ndof + ow[r]] = acc[s];
    }
    __syncthreads();
  }
  if (tr != 0 && tid < nr) {  // inverse row interchanges
    double2 *xr = x + (long long)tid * a.ndof;
    for (int j = k - 1; j >= 0; j--) {
      const int p = (int)a.piv[f.own0 + j] - 1;
      if (p != j) {
        const double2 t = xr[ow[j]];
        xr[ow[j]] = xr[ow[p]];
        xr[ow[p]] = t;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
void free_sparse(Ctx *c) {
  SparseLU *s = c->sparse;
  if (!s) return;
  void *ptrs[] = {s->d_fr,      s->d_own,     s->d_bnd,     s->d_ea,      s->d_lev_fronts,
                  s->d_ent_idx, s->d_ent_loc, s->d_fac,     s->d_piv,     s->d_work[0],
                  s->d_work[1], s->d_info};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (SpLane &ln : s->lane) {
    if (ln.dwork) cudaFree(ln.dwork);
    if (ln.d_getrf_info) cudaFree(ln.d_getrf_info);
    if (ln.par) cusolverDnDestroyParams(ln.par);
    if (ln.sol) cusolverDnDestroy(ln.sol);
    if (ln.blas) cublasDestroy(ln.blas);
    if (ln.done) cudaEventDestroy(ln.done);
    if (ln.st) cudaStreamDestroy(ln.st);
  }
  if (s->level_ready) cudaEventDestroy(s->level_ready);
  delete s;
  c->sparse = nullptr;
}

void sparse_info(const Ctx *c, long long *out) {
  const SparseLU *s = c->sparse;
  if (!s) {
    for (int i = 0; i < 7; i++) out[i] = 0;
    return;
  }
  plan_stats(s->fr, s->fac_elems, s->lev_work, out);
}

#define SPCK(expr, what)                                                   \
  do {                                                                     \
    cudaError_t e_ = (expr);                                               \
    if (e_ != cudaSuccess) {                                               \
      *msg = std::string("sparse solve: ") + (what) + ": " + cudaGetErrorString(e_); \
      return e_ == cudaErrorMemoryAllocation ? FEM25_ERR_ALLOC : FEM25_ERR_CUDA;     \
    }                                                                      \
  } while (0)

int sparse_factor(Ctx *c, const double *csr128, cudaStream_t st, std::string *msg) {
  if (!c->sparse) c->sparse = new SparseLU();
  SparseLU *s = c->sparse;
  s->factored = false;
  if (!s->analysed) {
    const int r = sparse_analyse(c, s, st, msg);
    if (r) return r;
  }
  if (!s->level_ready) {
    SPCK(cudaFuncSetAttribute(k_sp_factor_blk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(double2) * sp::kSmallN * sp::kNb)),
         "kernel attributes");
    SPCK(cudaEventCreateWithFlags(&s->level_ready, cudaEventDisableTiming), "events");
    for (SpLane &ln : s->lane) {
      SPCK(cudaStreamCreateWithFlags(&ln.st, cudaStreamNonBlocking), "streams");
      SPCK(cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming), "events");
      SPCK(cudaMalloc(&ln.d_getrf_info, sizeof(int)), "status");
      if (cusolverDnCreate(&ln.sol) != CUSOLVER_STATUS_SUCCESS ||
          cusolverDnCreateParams(&ln.par) != CUSOLVER_STATUS_SUCCESS ||
          cublasCreate(&ln.blas) != CUBLAS_STATUS_SUCCESS ||
          cusolverDnSetStream(ln.sol, ln.st) != CUSOLVER_STATUS_SUCCESS ||
          cublasSetStream(ln.blas, ln.st) != CUBLAS_STATUS_SUCCESS) {
        *msg = "sparse solve: cuSOLVER / cuBLAS handle creation failed";
        return FEM25_ERR_CUDA;
      }
    }
  }
  if (!s->d_fac) {
    SPCK(cudaMalloc(&s->d_fac, sizeof(double2) * std::max(s->fac_elems, 1LL)), "factor store");
    SPCK(cudaMalloc(&s->d_piv, sizeof(int64_t) * std::max(c->ndof, 1)), "pivots");
    SPCK(cudaMalloc(&s->d_work[0], sizeof(double2) * std::max(s->max_work, 1LL)), "work");
    SPCK(cudaMalloc(&s->d_work[1], sizeof(double2) * std::max(s->max_work, 1LL)), "work");
    SPCK(cudaMalloc(&s->d_info, sizeof(int)), "status");
  }
  SPCK(cudaMemsetAsync(s->d_info, 0, sizeof(int), st), "status");
  const double2 *csr = reinterpret_cast<const double2 *>(csr128);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  for (int l = s->nlevel - 1; l >= 0; l--) {
    double2 *W = s->d_work[l & 1], *Wc = s->d_work[(l + 1) & 1];
    const int nfl = (int)s->lev[l].size();
    const int *dfr = s->d_lev_fronts + s->lev_off[l];
    SPCK(cudaMemsetAsync(W, 0, sizeof(double2) * s->lev_work[l], st), "work");
    const long long ne = s->lev_ent0[l + 1] - s->lev_ent0[l];
    if (ne > 0) {
      const int grid = (int)std::min<long long>((ne + 255) / 256, (long long)nsm * 16);
      k_sp_assemble<<<grid, 256, 0, st>>>(ne, s->d_ent_idx + s->lev_ent0[l],
                                          s->d_ent_loc + s->lev_ent0[l], csr, W);
    }
    // more CTAs per front where the level has few fronts
    const unsigned ysplit = (unsigned)std::max(1, std::min(64, 2 * nsm / std::max(nfl, 1)));
    if (l + 1 < s->nlevel)
      for (int slot = 0; slot < 2; slot++)
        k_sp_extend_add<<<dim3(nfl, ysplit), 256, 0, st>>>(dfr, s->d_fr, s->d_ea, Wc, W, slot);
    SPCK(cudaGetLastError(), "assembly");
    // one CTA per front up to kSmallN rows; larger fronts: dense library calls
    const int nsmall = s->lev_nsmall[l];
    if (nsmall > 0) {
      const size_t sm = sizeof(double2) * (size_t)s->lev_nmax_small[l] * sp::kNb;
      k_sp_factor_blk<<<nsmall, sp::kFacThreads, sm, st>>>(dfr, nsmall, s->d_fr, W, s->d_piv,
                                                         s->d_info);
      SPCK(cudaGetLastError(), "small fronts");
    }
    std::vector<int> large(s->lev[l].begin() + nsmall, s->lev[l].end());
    // the level's large fronts spread over the lanes' streams, joined back
    // into the caller's stream before the factors are stored
    const int nl = (int)std::min<size_t>(large.size(), sp::kLanes);
    if (nl > 0) {
      SPCK(cudaEventRecord(s->level_ready, st), "events");
      for (int q = 0; q < nl; q++)
        SPCK(cudaStreamWaitEvent(s->lane[q].st, s->level_ready, 0), "events");
    }
    for (size_t q = 0; q < large.size(); q++) {
      const int t = large[q];
      SpLane &ln = s->lane[q % sp::kLanes];
      const SpFront &f = s->fr[t];
      const int64_t n = (int64_t)f.k + f.m, k = f.k, m = f.m;
      if (k == 0) continue;
      double2 *F = W + f.work0;
      size_t dbytes = 0, hbytes = 0;
      if (cusolverDnXgetrf_bufferSize(ln.sol, ln.par, k, k, CUDA_C_64F, F, n, CUDA_C_64F, &dbytes,
                                      &hbytes) != CUSOLVER_STATUS_SUCCESS) {
        *msg = "sparse solve: getrf workspace query failed";
        return FEM25_ERR_CUDA;
      }
      if (dbytes > ln.dwork_bytes) {
        // the lane's earlier calls may still use the old workspace
        SPCK(cudaStreamSynchronize(ln.st), "workspace");
        if (ln.dwork) SPCK(cudaFree(ln.dwork), "workspace");
        ln.dwork = nullptr;
        SPCK(cudaMalloc(&ln.dwork, dbytes), "workspace");
        ln.dwork_bytes = dbytes;
      }
      if (hbytes > ln.hwork.size()) ln.hwork.resize(hbytes);
      int64_t *ipiv = s->d_piv + f.own0;
      if (cusolverDnXgetrf(ln.sol, ln.par, k, k, CUDA_C_64F, F, n, ipiv, CUDA_C_64F, ln.dwork,
                           dbytes, hbytes ? ln.hwork.data() : nullptr, hbytes,
                           ln.d_getrf_info) != CUSOLVER_STATUS_SUCCESS) {
        *msg = "sparse solve: getrf failed";
        return FEM25_ERR_CUDA;
      }
      // a zero pivot of this front: recorded as the front's id in the status word
      k_sp_getrf_status<<<1, 1, 0, ln.st>>>(ln.d_getrf_info, s->d_info, t);
      if (m > 0) {
        k_sp_laswp<<<(int)std::min<int64_t>((m + 127) / 128, 1024), 128, 0, ln.st>>>(
            F, (int)n, (int)k, (int)k, (int)n, ipiv);
        SPCK(cudaGetLastError(), "laswp");
        const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0),
                              mone = make_cuDoubleComplex(-1.0, 0.0);
        cuDoubleComplex *A = reinterpret_cast<cuDoubleComplex *>(F);
        if (cublasZtrsm(ln.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                        CUBLAS_DIAG_UNIT, (int)k, (int)m, &one, A, (int)n, A + k * n, (int)n) ||
            cublasZtrsm(ln.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                        CUBLAS_DIAG_NON_UNIT, (int)m, (int)k, &one, A, (int)n, A + k, (int)n) ||
            cublasZgemm(ln.blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)m, (int)m, (int)k, &mone, A + k,
                        (int)n, A + k * n, (int)n, &one, A + k + k * n, (int)n)) {
          *msg = "sparse solve: trsm / gemm failed";
          return FEM25_ERR_CUDA;
        }
      }
    }
    for (int q = 0; q < nl; q++) {
      SPCK(cudaEventRecord(s->lane[q].done, s->lane[q].st), "events");
      SPCK(cudaStreamWaitEvent(st, s->lane[q].done, 0), "events");
    }
    k_sp_store<<<dim3(nfl, ysplit), 256, 0, st>>>(dfr, s->d_fr, W, s->d_fac);
    SPCK(cudaGetLastError(), "factor store");
  }
  // zero pivots of any front
  int info = 0;
  SPCK(cudaMemcpyAsync(&info, s->d_info, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
  SPCK(cudaStreamSynchronize(st), "factorisation");
  if (info != 0) {
    *msg = "sparse solve: zero pivot in front " + std::to_string(info - 1) +
           " (matrix singular to working precision)";
    return FEM25_ERR_ARG;
  }
  s->factored = true;
  return 0;
}

// the level-by-level launches of one solve, R right-hand sides per CTA
template <int R>
static void sparse_solve_levels(const SparseLU *s, SolveArgs a, cudaStream_t st) {
  const unsigned nchunk = (unsigned)((a.nrhs + R - 1) / R);
  auto tiles = [](int rows) { return (unsigned)std::max(1, (rows + sp::kThreads - 1) / sp::kThreads); };
  for (int l = s->nlevel - 1; l >= 0; l--) {  // forward, from the leaves
    a.fronts = s->d_lev_fronts + s->lev_off[l];
    const unsigned nfl = (unsigned)s->lev[l].size();
    k_sp_solve_fwd<R><<<dim3(nfl, nchunk), sp::kThreads, 0, st>>>(a);
    if (s->lev_mmax[l] > 0)
      k_sp_solve_rect<R><<<dim3(nfl, tiles(s->lev_mmax[l]), nchunk), sp::kThreads, 0, st>>>(a, 1);
  }
  for (int l = 0; l < s->nlevel; l++) {  // backward, from the root
    a.fronts = s->d_lev_fronts + s->lev_off[l];
    const unsigned nfl = (unsigned)s->lev[l].size();
    if (s->lev_mmax[l] > 0)
      k_sp_solve_rect<R><<<dim3(nfl, tiles(s->lev_kmax[l]), nchunk), sp::kThreads, 0, st>>>(a, 0);
    k_sp_solve_bwd<R><<<dim3(nfl, nchunk), sp::kThreads, 0, st>>>(a);
  }
}

int sparse_solve(Ctx *c, int nrhs, int trans, double *rhs, cudaStream_t st, std::string *msg) {
  SparseLU *s = c->sparse;
  if (!s || !s->factored) {
    *msg = "sparse solve: no factorisation (call fem25_sparse_factor_dev first)";
    return FEM25_ERR_ARG;
  }
  SolveArgs a{nullptr, s->d_fr, s->d_own, s->d_bnd, s->d_fac, s->d_piv,
              reinterpret_cast<double2 *>(rhs), c->ndof, nrhs, trans};
  if (nrhs == 1)
    sparse_solve_levels<1>(s, a, st);
  else
    sparse_solve_levels<sp::kRhsPerCta>(s, a, st);
  SPCK(cudaGetLastError(), "solve");
  return 0;
}

}  // namespace fem25
