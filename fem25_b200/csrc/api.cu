// C ABI of libfem25gpu (include/fem25gpu.h): argument checks, device
// memory, context life cycle and the orchestration of the kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <map>

#include "ctx.cuh"

using namespace fem25;

struct fem25_graph {
  HostGraph g;
};
struct fem25_ctx {
  Ctx c;
};

namespace {

// true while stream st records into a CUDA graph
bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

int fail(Ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  std::fprintf(stderr, "fem25gpu: %s\n", msg.c_str());
  return code;
}

int cuda_fail(Ctx *c, cudaError_t e, const char *where) {
  return fail(c, FEM25_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call, where)                              \
  do {                                               \
    cudaError_t _e = (call);                         \
    if (_e != cudaSuccess) return cuda_fail(c, _e, where); \
  } while (0)

template <class T>
cudaError_t dalloc_copy(T **d, const T *h, size_t n) {
  cudaError_t e = cudaMalloc((void **)d, sizeof(T) * (n ? n : 1));
  if (e) return e;
  if (n) e = cudaMemcpy(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
  return e;
}

int check_mesh(const fem25_mesh *m, std::string *msg) {
  if (!m || !m->ieng || !m->cdomain || !m->cnnpg || !m->xlocs || !m->zlocs || !m->xd || !m->zd ||
      !m->ecoeff || !m->dens) {
    *msg = "mesh: null array";
    return FEM25_ERR_ARG;
  }
  if (m->nelem <= 0 || m->nnpg <= 0) {
    *msg = "mesh: empty";
    return FEM25_ERR_ARG;
  }
  if (m->nord != kNord) {
    *msg = "mesh: only NORD = 4 (5x5 GLL nodes) is built";
    return FEM25_ERR_UNSUPPORTED;
  }
  if (m->ldisp && (!m->qp || !m->qs)) {
    *msg = "mesh: dispersive media (ldisp = 1) need QP and QS";
    return FEM25_ERR_ARG;
  }
  for (int e = 0; e < m->nelem; e++) {
    for (int a = 0; a < 4; a++) {
      int p = m->ieng[4 * (size_t)e + a];
      if (p < 1 || p > m->nnpg) {
        *msg = "mesh: IENG entry out of range";
        return FEM25_ERR_ARG;
      }
    }
    char d = m->cdomain[e];
    if (d != 'I' && d != 'E' && d != 'A') {
      *msg = "mesh: CDOMAIN must be 'I', 'E' or 'A'";
      return FEM25_ERR_ARG;
    }
  }
  return FEM25_OK;
}

void free_ctx(Ctx *c) {
  void *ptrs[] = {c->dt.xigll, c->dt.wts, c->dt.shl, c->dt.sf, c->dt.dsf, c->d_ieng, c->d_cdomain,
                  c->d_x, c->d_z, c->d_xd, c->d_zd, c->d_lam, c->d_mu, c->d_rho, c->d_lm,
                  c->d_irptr, c->d_jcptr, c->d_cnp, c->d_elemmat, c->d_gptr, c->d_glist, c->d_err,
                  c->d_brptr, c->d_brow, c->d_basis, c->d_ebasis, c->d_bgptr, c->d_bglist,
                  c->d_pml_elems, c->d_pml_idx, c->d_pgptr, c->d_pglist, c->d_pml_emat,
                  c->d_pml_delta, c->d_jcsc, c->d_icsc, c->d_rg_anchor, c->d_mconn,
                  c->d_elem_wts, c->d_fmat, c->d_cadj_col0, c->d_cadj_pair_col, c->d_cadj_pair_elem,
                  c->d_cadj_dptr, c->d_cadj_dent, c->d_cadj_w, c->d_nonpml, c->d_cdist, c->d_prim, c->d_desc,
                  c->d_tc_tab, c->d_qp, c->d_qs, c->d_cov, c->d_cov_ops, c->d_cov_opptr,
                  c->d_cov_tx, c->d_cov_node, c->d_cov_exps, c->d_maskg, c->d_avg_work, c->d_post_mrdof,
                  c->d_post_bits, c->d_hvec, c->d_hgrad};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto &e : c->drv_ev)
    if (e) cudaEventDestroy(e);
  if (c->copy_st) cudaStreamDestroy(c->copy_st);
  free_dense(c);
  free_sparse(c);
}

int read_err_word(Ctx *c, cudaStream_t st) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, st), "error word");
  CK(cudaStreamSynchronize(st), "synchronize");
  if (h > 0) {
    char buf[128];
    std::snprintf(buf, sizeof buf, "element %d: Jacobian undefined or negative", h);
    cudaMemsetAsync(c->d_err, 0, sizeof(int), st);
    return fail(c, FEM25_ERR_JACOBIAN, buf);
  }
  if (h <= -1000000) {
    // a bounded wait of a tensor-core gradient kernel ran out (-1000001..:
    // pointwise form, -2000001..: covariance form; the last digit names the
    // hand-off); the kernel drained its schedule and returned
    char buf[200];
    std::snprintf(buf, sizeof buf,
                  "gradient: a tensor-core pipeline wait timed out (code %d); results of that "
                  "launch, and covariances accumulated since the last finalize, are discarded",
                  h);
    cudaMemsetAsync(c->d_err, 0, sizeof(int), st);
    c->cov_pending = false;  // the next accumulation overwrites the sums
    return fail(c, FEM25_ERR_CUDA, buf);
  }
  if (h < 0) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), st);
    return fail(c, FEM25_ERR_PATTERN, "element entry without a CSR / CSC slot");
  }
  return FEM25_OK;
}


int upload_model(Ctx *c, const double *ecoeff, const double *dens) {
  const size_t n = c->nnpg;
  for (size_t p = 0; p < n; p++)
    if (!(dens[p] > 0.0) || !(ecoeff[n + p] >= 0.0) || !(ecoeff[p] + 2.0 * ecoeff[n + p] > 0.0))
      return fail(c, FEM25_ERR_ARG, "model: density must be > 0, mu >= 0, lambda + 2 mu > 0");
  CK(cudaMemcpy(c->d_lam, ecoeff, sizeof(double) * n, cudaMemcpyHostToDevice), "model upload");
  CK(cudaMemcpy(c->d_mu, ecoeff + n, sizeof(double) * n, cudaMemcpyHostToDevice), "model upload");
  CK(cudaMemcpy(c->d_rho, dens, sizeof(double) * n, cudaMemcpyHostToDevice), "model upload");
  c->basis_valid = false;
  return FEM25_OK;
}

int ensure_plain(Ctx *c, cudaStream_t st) {
  if (c->d_gptr) return FEM25_OK;
  if (capturing(st))
    return fail(c, FEM25_ERR_ARG,
                "assemble: the gather map is built on the first call (synchronously); make one "
                "uncaptured call before capturing");
  CK(cudaMalloc(&c->d_elemmat, sizeof(double2) * 9 * (size_t)c->nelem * kNab), "element matrices");
  CK(build_gather_map(c, st), "gather map");
  return read_err_word(c, st);
}

int ensure_batch(Ctx *c, cudaStream_t st) {
  if (c->mesh_scalars.ldisp)
    return fail(c, FEM25_ERR_UNSUPPORTED,
                "batch: dispersive media have frequency-dependent complex velocities "
                "(no per-mesh affine basis); use fem25_assemble_dev");
  if (c->bcsr.nblocks >= (1LL << 28))
    return fail(c, FEM25_ERR_UNSUPPORTED, "batch: more than 2^28 node blocks");
  if ((!c->d_bgptr || !c->basis_valid) && capturing(st))
    return fail(c, FEM25_ERR_ARG,
                "batch: the affine basis is built on the first call (synchronously); make one "
                "uncaptured call before capturing");
  if (!c->d_bgptr) {
    CK(build_batch_structures(c, st), "batch structures");
    int r = read_err_word(c, st);
    if (r) return r;
  }
  if (!c->basis_valid) {
    CK(build_basis(c, st), "basis");
    int r = read_err_word(c, st);
    if (r) return r;
    c->basis_valid = true;
  }
  return FEM25_OK;
}

// Chunking of fem25_asmble_driver: up to 16 element ranges of at least one
// wave of CTAs each; the CSR rows are the DOFs, and row r is complete once
// the last element holding DOF r (GENID numbers DOFs in element order, so
// rows complete nearly in order) has been computed.
int ensure_driver_plan(Ctx *c) {
  if (c->copy_st) return FEM25_OK;
  const int nch = std::max(1, std::min(16, c->nelem / 148));
  std::vector<int> last(c->ndof, -1);
  for (int e = 0; e < c->nelem; e++)
    for (int k = 0; k < 3 * kNen; k++) {
      const int d = c->h_lm[(size_t)e * 3 * kNen + k];
      if (d > 0) last[d - 1] = e;
    }
  c->drv_elem.assign(nch + 1, 0);
  c->drv_row.assign(nch + 1, 0);
  for (int k = 0; k <= nch; k++) c->drv_elem[k] = (int)((long long)k * c->nelem / nch);
  int r = 0;
  for (int k = 1; k <= nch; k++) {
    while (r < c->ndof && last[r] < c->drv_elem[k]) r++;
    c->drv_row[k] = r;
  }
  if (c->drv_row[nch] != c->ndof)
    return fail(c, FEM25_ERR_PATTERN, "asmble_driver: DOF outside every element");
  c->drv_ev.assign(nch, nullptr);
  for (auto &e : c->drv_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  CK(cudaStreamCreateWithFlags(&c->copy_st, cudaStreamNonBlocking), "copy stream");
  return FEM25_OK;
}

int ensure_refgrad(Ctx *c) {
  if (c->refgrad_ready) return FEM25_OK;
  if (c->mesh_scalars.ldisp)
    return fail(c, FEM25_ERR_UNSUPPORTED, "gradient: dispersive media are not supported");
  fem25_mesh m = c->mesh_scalars;
  m.ieng = c->h_ieng.data();
  m.cdomain = c->h_cdomain.data();
  m.cnnpg = c->h_cnnpg.data();
  m.xlocs = c->h_x.data();
  m.zlocs = c->h_z.data();
  std::string msg;
  int r = build_ref_grad(&m, c->h_lm.data(), &c->rg, &msg);
  if (r) return fail(c, r, msg);
  CK(dalloc_copy(&c->d_jcsc, c->rg.jcsc.data(), c->rg.jcsc.size()), "ref grad");
  CK(dalloc_copy(&c->d_icsc, c->rg.icsc.data(), c->rg.icsc.size()), "ref grad");
  CK(dalloc_copy(&c->d_rg_anchor, c->rg.anchor_of_col.data(), c->rg.anchor_of_col.size()), "ref grad");
  CK(dalloc_copy(&c->d_mconn, c->rg.mconn.data(), c->rg.mconn.size()), "ref grad");
  CK(dalloc_copy(&c->d_maskg, c->rg.maskg.data(), c->rg.maskg.size()), "ref grad");
  CK(cudaMalloc(&c->d_avg_work, sizeof(double) * 2 * (size_t)std::max(c->rg.nnpinv, 1)),
     "ref grad");
  CK(dalloc_copy(&c->d_elem_wts, c->rg.elem_wts.data(), c->rg.elem_wts.size()), "ref grad");
  CK(cudaMalloc(&c->d_fmat, sizeof(float2) * (c->rg.nz ? c->rg.nz : 1)), "ref grad");
  c->refgrad_ready = true;
  return FEM25_OK;
}

}  // namespace

extern "C" {

int fem25_graph_build(const fem25_mesh *m, fem25_graph **out) {
  std::string msg;
  if (!out) return FEM25_ERR_ARG;
  int r = check_mesh(m, &msg);
  if (r) return fail(nullptr, r, msg);
  fem25_graph *g = new fem25_graph();
  r = build_graph(m, &g->g, &msg);
  if (r) {
    delete g;
    return fail(nullptr, r, msg);
  }
  *out = g;
  return FEM25_OK;
}

int fem25_graph_info(const fem25_graph *g, int *nnp, int *ndof, long long *nzero) {
  if (!g) return FEM25_ERR_ARG;
  if (nnp) *nnp = g->g.nnp;
  if (ndof) *ndof = g->g.ndof;
  if (nzero) *nzero = g->g.nzero;
  return FEM25_OK;
}

int fem25_graph_copy(const fem25_graph *g, int *ien, int *lm, int *irptr, int *jcptr, char *cnp) {
  if (!g) return FEM25_ERR_ARG;
  const HostGraph &h = g->g;
  if (ien) std::memcpy(ien, h.ien.data(), sizeof(int) * h.ien.size());
  if (lm) std::memcpy(lm, h.lm.data(), sizeof(int) * h.lm.size());
  if (irptr) std::memcpy(irptr, h.irptr.data(), sizeof(int) * h.irptr.size());
  if (jcptr) std::memcpy(jcptr, h.jcptr.data(), sizeof(int) * h.jcptr.size());
  if (cnp) std::memcpy(cnp, h.cnp.data(), h.cnp.size());
  return FEM25_OK;
}

void fem25_graph_free(fem25_graph *g) { delete g; }
// FNV-1a 64 over the mesh arrays the graph depends on
static uint64_t mesh_fingerprint(const fem25_mesh *m) {
  uint64_t h = 1469598103934665603ULL;
  auto mix = [&](const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ULL;
  };
  mix(&m->nelem, sizeof(int));
  mix(&m->nnpg, sizeof(int));
  mix(&m->nord, sizeof(int));
  mix(m->ieng, sizeof(int) * 4 * (size_t)m->nelem);
  mix(m->cdomain, (size_t)m->nelem);
  mix(m->cnnpg, 2 * (size_t)m->nnpg);
  mix(m->xlocs, sizeof(double) * (size_t)m->nnpg);
  mix(m->zlocs, sizeof(double) * (size_t)m->nnpg);
  return h;
}

static const char kGraphMagic[8] = {'F', 'E', 'M', '2', '5', 'G', 'R', '1'};

int fem25_graph_save(const fem25_graph *g, const fem25_mesh *m, const char *path) {
  if (!g || !m || !path) return FEM25_ERR_ARG;
  std::string msg;
  int r = check_mesh(m, &msg);
  if (r) return fail(nullptr, r, msg);
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(nullptr, FEM25_ERR_ARG, std::string("graph save: cannot open ") + path);
  const HostGraph &h = g->g;
  const uint64_t fp = mesh_fingerprint(m);
  const int hdr[3] = {h.nelem, h.nnp, h.ndof};
  bool ok = std::fwrite(kGraphMagic, 1, 8, f) == 8 && std::fwrite(&fp, 8, 1, f) == 1 &&
            std::fwrite(hdr, sizeof(int), 3, f) == 3 && std::fwrite(&h.nzero, 8, 1, f) == 1;
  auto put = [&](const void *p, size_t sz, size_t n) {
    ok = ok && (n == 0 || std::fwrite(p, sz, n, f) == n);
  };
  put(h.ien.data(), sizeof(int), h.ien.size());
  put(h.lm.data(), sizeof(int), h.lm.size());
  put(h.irptr.data(), sizeof(int), h.irptr.size());
  put(h.jcptr.data(), sizeof(int), h.jcptr.size());
  put(h.cnp.data(), 1, h.cnp.size());
  ok = (std::fclose(f) == 0) && ok;
  return ok ? FEM25_OK : fail(nullptr, FEM25_ERR_ARG, "graph save: write failed");
}

int fem25_graph_load(const fem25_mesh *m, const char *path, fem25_graph **out) {
  if (!m || !path || !out) return FEM25_ERR_ARG;
  *out = nullptr;
  std::string msg;
  int r = check_mesh(m, &msg);
  if (r) return fail(nullptr, r, msg);
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(nullptr, FEM25_ERR_ARG, std::string("graph load: cannot open ") + path);
  char magic[8];
  uint64_t fp = 0;
  int hdr[3];
  long long nz = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kGraphMagic, 8) == 0 &&
            std::fread(&fp, 8, 1, f) == 1 && std::fread(hdr, sizeof(int), 3, f) == 3 &&
            std::fread(&nz, 8, 1, f) == 1;
  if (!ok || fp != mesh_fingerprint(m) || hdr[0] != m->nelem || hdr[2] <= 0 || nz <= 0) {
    std::fclose(f);
    return fail(nullptr, FEM25_ERR_GRAPH, "graph load: file does not belong to this mesh");
  }
  fem25_graph *g = new fem25_graph();
  HostGraph &h = g->g;
  h.nelem = hdr[0];
  h.nnp = hdr[1];
  h.ndof = hdr[2];
  h.nzero = nz;
  h.ien.resize((size_t)kNen * h.nelem);
  h.lm.resize((size_t)3 * kNen * h.nelem);
  h.irptr.resize((size_t)h.ndof + 1);
  h.jcptr.resize((size_t)nz);
  h.cnp.resize((size_t)h.ndof);
  auto get = [&](void *p, size_t sz, size_t n) { ok = ok && std::fread(p, sz, n, f) == n; };
  get(h.ien.data(), sizeof(int), h.ien.size());
  get(h.lm.data(), sizeof(int), h.lm.size());
  get(h.irptr.data(), sizeof(int), h.irptr.size());
  get(h.jcptr.data(), sizeof(int), h.jcptr.size());
  get(h.cnp.data(), 1, h.cnp.size());
  std::fclose(f);
  if (!ok || h.irptr[0] != 1 || h.irptr[h.ndof] != nz + 1) {
    delete g;
    return fail(nullptr, FEM25_ERR_GRAPH, "graph load: truncated or corrupt file");
  }
  *out = g;
  return FEM25_OK;
}

int fem25_create(const fem25_mesh *m, int ndof, long long nzero, const int *lm, const int *irptr,
                 const int *jcptr, const char *cnp, int device, fem25_ctx **out) {
  std::string msg;
  if (!out) return FEM25_ERR_ARG;
  *out = nullptr;
  int r = check_mesh(m, &msg);
  if (r) return fail(nullptr, r, msg);
  if (!lm || !irptr || !jcptr || !cnp || ndof <= 0 || nzero <= 0)
    return fail(nullptr, FEM25_ERR_ARG, "create: graph arrays missing");
  if (nzero > 2147483647LL) return fail(nullptr, FEM25_ERR_ARG, "create: NZERO exceeds int32");
  if (irptr[0] != 1 || irptr[ndof] - 1 != nzero)
    return fail(nullptr, FEM25_ERR_ARG, "create: IRPTR inconsistent with NZERO");
  for (size_t k = 0; k < (size_t)3 * kNen * m->nelem; k++)
    if (lm[k] < 0 || lm[k] > ndof) return fail(nullptr, FEM25_ERR_ARG, "create: LM out of range");
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || device < 0 || device >= ndev)
    return fail(nullptr, FEM25_ERR_CUDA, "create: no such CUDA device");
  fem25_ctx *h = new fem25_ctx();
  Ctx *c = &h->c;
  c->device = device;
  if ((ce = cudaSetDevice(device))) {
    delete h;
    return fail(nullptr, FEM25_ERR_CUDA, cudaGetErrorString(ce));
  }
  c->mesh_scalars = *m;
  c->mesh_scalars.ieng = nullptr;
  c->mesh_scalars.cdomain = nullptr;
  c->mesh_scalars.cnnpg = nullptr;
  c->mesh_scalars.xlocs = c->mesh_scalars.zlocs = c->mesh_scalars.xd = c->mesh_scalars.zd = nullptr;
  c->mesh_scalars.ecoeff = c->mesh_scalars.dens = nullptr;
  c->mesh_scalars.qp = c->mesh_scalars.qs = nullptr;
  c->nelem = m->nelem;
  c->nnpg = m->nnpg;
  c->ndof = ndof;
  c->nzero = nzero;
  c->h_cdomain.assign(m->cdomain, m->cdomain + m->nelem);
  c->h_cnnpg.assign(m->cnnpg, m->cnnpg + 2 * (size_t)m->nnpg);
  c->h_x.assign(m->xlocs, m->xlocs + m->nnpg);
  c->h_z.assign(m->zlocs, m->zlocs + m->nnpg);
  c->h_ieng.assign(m->ieng, m->ieng + 4 * (size_t)m->nelem);
  c->h_lm.assign(lm, lm + 3 * (size_t)kNen * m->nelem);
  c->h_irptr.assign(irptr, irptr + ndof + 1);
  r = build_block_csr(ndof, nzero, irptr, jcptr, &c->bcsr, &msg);
  if (r) {
    fail(c, r, msg);
    free_ctx(c);
    delete h;
    return r;
  }
  build_tables(&c->tab);
  auto setup = [&]() -> int {
    CK(dalloc_copy(&c->dt.xigll, c->tab.xigll, kNint), "tables");
    CK(dalloc_copy(&c->dt.wts, c->tab.wts, kNint), "tables");
    CK(dalloc_copy(&c->dt.shl, c->tab.shl, 3 * kNen * kNq), "tables");
    CK(dalloc_copy(&c->dt.sf, &c->tab.sf[0][0], 4 * kNq), "tables");
    CK(dalloc_copy(&c->dt.dsf, &c->tab.dsf[0][0][0], 8 * kNq), "tables");
    CK(dalloc_copy(&c->d_ieng, reinterpret_cast<const int4 *>(m->ieng), m->nelem), "mesh");
    CK(dalloc_copy(&c->d_cdomain, m->cdomain, m->nelem), "mesh");
    CK(dalloc_copy(&c->d_x, m->xlocs, m->nnpg), "mesh");
    CK(dalloc_copy(&c->d_z, m->zlocs, m->nnpg), "mesh");
    CK(dalloc_copy(&c->d_xd, m->xd, m->nnpg), "mesh");
    CK(dalloc_copy(&c->d_zd, m->zd, m->nnpg), "mesh");
    CK(cudaMalloc(&c->d_lam, sizeof(double) * m->nnpg), "mesh");
    CK(cudaMalloc(&c->d_mu, sizeof(double) * m->nnpg), "mesh");
    CK(cudaMalloc(&c->d_rho, sizeof(double) * m->nnpg), "mesh");
    int rr = upload_model(c, m->ecoeff, m->dens);
    if (rr) return rr;
    if (m->ldisp) {
      CK(dalloc_copy(&c->d_qp, m->qp, m->nnpg), "mesh");
      CK(dalloc_copy(&c->d_qs, m->qs, m->nnpg), "mesh");
    }
    CK(dalloc_copy(&c->d_lm, lm, 3 * (size_t)kNen * m->nelem), "graph");
    CK(dalloc_copy(&c->d_irptr, irptr, (size_t)ndof + 1), "graph");
    CK(dalloc_copy(&c->d_jcptr, jcptr, (size_t)nzero), "graph");
    CK(dalloc_copy(&c->d_cnp, cnp, (size_t)ndof), "graph");
    CK(cudaMalloc(&c->d_err, sizeof(int)), "error word");
    CK(cudaMemset(c->d_err, 0, sizeof(int)), "error word");
    std::vector<int> nonpml;
    for (int e = 0; e < m->nelem; e++)
      if (m->cdomain[e] != 'A') nonpml.push_back(e);
    c->n_nonpml = (int)nonpml.size();
    CK(dalloc_copy(&c->d_nonpml, nonpml.data(), nonpml.size()), "element lists");
    c->mv.nelem = m->nelem;
    c->mv.nnpg = m->nnpg;
    c->mv.ieng = c->d_ieng;
    c->mv.cdomain = c->d_cdomain;
    c->mv.x = c->d_x;
    c->mv.z = c->d_z;
    c->mv.xd = c->d_xd;
    c->mv.zd = c->d_zd;
    c->mv.lam = c->d_lam;
    c->mv.mu = c->d_mu;
    c->mv.rho = c->d_rho;
    c->mv.qp = c->d_qp;
    c->mv.qs = c->d_qs;
    CK(check_jacobians(c, 0), "jacobian check");
    return read_err_word(c, 0);
  };
  r = setup();
  if (r) {
    free_ctx(c);
    delete h;
    return r;
  }
  *out = h;
  return FEM25_OK;
}

void fem25_destroy(fem25_ctx *h) {
  if (!h) return;
  cudaSetDevice(h->c.device);
  cudaDeviceSynchronize();
  free_ctx(&h->c);
  delete h;
}

int fem25_last_error(const fem25_ctx *h, char *buf, int n) {
  if (!h || !buf || n <= 0) return FEM25_ERR_ARG;
  std::snprintf(buf, n, "%s", h->c.err.c_str());
  return FEM25_OK;
}

int fem25_sizes(const fem25_ctx *h, int *ndof, long long *nzero, long long *nblocks) {
  if (!h) return FEM25_ERR_ARG;
  if (ndof) *ndof = h->c.ndof;
  if (nzero) *nzero = h->c.nzero;
  if (nblocks) *nblocks = h->c.bcsr.nblocks;
  return FEM25_OK;
}

int fem25_update_model(fem25_ctx *h, const double *ecoeff, const double *dens) {
  if (!h || !ecoeff || !dens) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  return upload_model(c, ecoeff, dens);
}

int fem25_assemble_dev(fem25_ctx *h, char cftype, double freq, double py, double *csr128,
                       float *csr64, void *stream) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (cftype != 'S' && cftype != 'B') return fail(c, FEM25_ERR_ARG, "assemble: CFTYPE must be 'S' or 'B'");
  if (!(freq > 0.0)) return fail(c, FEM25_ERR_ARG, "assemble: FREQ must be > 0");
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_plain(c, st);
  if (r) return r;
  if (c->prof) CK(cudaEventRecord(c->ev[2], st), "event");
  if (c->plain_fma)
    CK(launch_elem_plain_fma(c, cftype, freq, py, 0, c->nelem, st), "element kernel (FMA)");
  else
    CK(launch_elem_plain(c, cftype, freq, py, 0, c->nelem, st), "element kernel");
  CK(launch_gather_plain(c, csr128, csr64, 0, c->nzero, st), "gather kernel");
  if (c->prof) CK(cudaEventRecord(c->ev[3], st), "event");
  return FEM25_OK;
}

int fem25_asmble_driver(fem25_ctx *h, int nzloc, char cftype, double freq, double py,
                        float *cdist) {
  if (!h || !cdist) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if ((long long)nzloc != c->nzero) return fail(c, FEM25_ERR_ARG, "asmble_driver: NZLOC != NZERO");
  if (cftype != 'S' && cftype != 'B')
    return fail(c, FEM25_ERR_ARG, "asmble_driver: CFTYPE must be 'S' or 'B'");
  if (!(freq > 0.0)) return fail(c, FEM25_ERR_ARG, "asmble_driver: FREQ must be > 0");
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_plain(c, nullptr);
  if (r) return r;
  if (!c->d_cdist) CK(cudaMalloc(&c->d_cdist, sizeof(float2) * (size_t)nzloc), "cdist buffer");
  r = ensure_driver_plan(c);
  if (r) return r;
  // every chunk's element matrices and gather are enqueued first, then the
  // host copies follow the chunks as they complete (a pageable destination
  // makes each copy synchronous for the host, the GPU keeps computing)
  cudaStream_t st = nullptr;
  const int nch = (int)c->drv_elem.size() - 1;
  for (int k = 0; k < nch; k++) {
    const long long nz0 = c->h_irptr[c->drv_row[k]] - 1, nz1 = c->h_irptr[c->drv_row[k + 1]] - 1;
    CK(launch_elem_plain(c, cftype, freq, py, c->drv_elem[k], c->drv_elem[k + 1], st),
       "element kernel");
    CK(launch_gather_plain(c, nullptr, (float *)c->d_cdist, nz0, nz1, st), "gather kernel");
    CK(cudaEventRecord(c->drv_ev[k], st), "event");
  }
  for (int k = 0; k < nch; k++) {
    const long long nz0 = c->h_irptr[c->drv_row[k]] - 1, nz1 = c->h_irptr[c->drv_row[k + 1]] - 1;
    if (nz1 <= nz0) continue;
    CK(cudaStreamWaitEvent(c->copy_st, c->drv_ev[k], 0), "event");
    CK(cudaMemcpyAsync(cdist + 2 * nz0, c->d_cdist + nz0, sizeof(float2) * (size_t)(nz1 - nz0),
                       cudaMemcpyDeviceToHost, c->copy_st),
       "cdist copy");
  }
  CK(cudaStreamSynchronize(c->copy_st), "cdist copy");
  return read_err_word(c, 0);
}

int fem25_assemble_batch_dev(fem25_ctx *h, int n, const char *cftype, const double *freq,
                             const double *py, double *ring_base, long long slot_stride,
                             int nslots, void *stream) {
  if (!h || !cftype || !freq || !py || !ring_base || n <= 0 || nslots <= 0) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (slot_stride < 2 * c->nzero || (slot_stride & 1))
    return fail(c, FEM25_ERR_ARG, "batch: slot stride must be even and >= 2*NZERO");
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_batch(c, st);
  if (r) return r;
  // distinct (omega, cftype) -> PML delta slots
  std::map<std::pair<double, char>, int> slots;
  std::vector<std::pair<double, char>> order;
  for (int k = 0; k < n; k++) {
    if (cftype[k] != 'S' && cftype[k] != 'B')
      return fail(c, FEM25_ERR_ARG, "batch: CFTYPE must be 'S' or 'B'");
    if (!(freq[k] > 0.0)) return fail(c, FEM25_ERR_ARG, "batch: FREQ must be > 0");
    auto key = std::make_pair(freq[k], cftype[k]);
    if (!slots.count(key)) {
      slots[key] = (int)order.size();
      order.push_back(key);
    }
  }
  const int nps = (int)order.size();
  if (c->npml_blocks > 0 && nps > c->pml_delta_cap) {
    if (capturing(st))
      return fail(c, FEM25_ERR_ARG,
                  "batch: more distinct (FREQ, CFTYPE) pairs than any earlier call; make one "
                  "uncaptured call of this size before capturing");
    CK(cudaStreamSynchronize(st), "synchronize");
    if (c->d_pml_delta) cudaFree(c->d_pml_delta);
    CK(cudaMalloc(&c->d_pml_delta, sizeof(double2) * 9 * (size_t)c->npml_blocks * nps), "pml delta");
    c->pml_delta_cap = nps;
  }
  for (int k = 0; k < nps; k++) {
    PmlParams pp = pml_params(c, order[k].second, order[k].first);
    CK(build_pml_delta(c, pp, k, st), "pml delta");
  }
  std::vector<SysParam> sys(n);
  for (int k = 0; k < n; k++) {
    double omega = 6.2831853071795862 * freq[k];
    sys[k].w2 = omega * omega;
    sys[k].wpy = omega * py[k];
    sys[k].pml_slot = slots[std::make_pair(freq[k], cftype[k])];
    sys[k].pad = 0;
  }
  if (c->prof) CK(cudaEventRecord(c->ev[0], st), "event");
  CK(launch_stream_batch(c, n, sys.data(), ring_base, slot_stride, nslots, st), "stream kernel");
  if (c->prof) CK(cudaEventRecord(c->ev[1], st), "event");
  return FEM25_OK;
}

int fem25_sync_status(fem25_ctx *h, void *stream) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  return read_err_word(c, (cudaStream_t)stream);
}

int fem25_plain_fma(fem25_ctx *h, int enable) {
  if (!h) return FEM25_ERR_ARG;
  h->c.plain_fma = enable != 0;
  return FEM25_OK;
}

int fem25_test_waits(fem25_ctx *h, long long limit_cycles, int inject) {
  if (!h || (inject != 0 && inject != 1)) return FEM25_ERR_ARG;
  h->c.wait_limit = limit_cycles > 0 ? limit_cycles : 0;
  h->c.wait_inject = inject;
  return FEM25_OK;
}

int fem25_tuning(const fem25_ctx *h, int *stream_variant, int *grad_tile) {
  if (!h) return FEM25_ERR_ARG;
  if (stream_variant) *stream_variant = h->c.stream_variant;
  if (grad_tile) *grad_tile = h->c.grad_tile;
  return FEM25_OK;
}

int fem25_profile_enable(fem25_ctx *h, int enable) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  for (auto &e : c->ev)
    if (!e) CK(cudaEventCreate(&e), "event");
  c->prof = enable != 0;
  return FEM25_OK;
}

int fem25_profile_ms(fem25_ctx *h, int which, double *ms) {
  if (!h || !ms || which < 0 || which > 1) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (!c->ev[2 * which]) return fail(c, FEM25_ERR_ARG, "profiling not enabled");
  CK(cudaEventSynchronize(c->ev[2 * which + 1]), "event");
  float t = 0.f;
  CK(cudaEventElapsedTime(&t, c->ev[2 * which], c->ev[2 * which + 1]), "event");
  *ms = t;
  return FEM25_OK;
}

int fem25_peff_dev(fem25_ctx *h, int nsrc, const float *a_loc, const float *ue, float *peff,
                   void *stream) {
  if (!h || !a_loc || !ue || !peff || nsrc <= 0) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  CK(launch_peff(c, nsrc, a_loc, ue, peff, (cudaStream_t)stream), "peff");
  return FEM25_OK;
}

int fem25_dense_factor_dev(fem25_ctx *h, const double *csr128, void *stream) {
  if (!h || !csr128) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (c->ndof > FEM25_DENSE_MAX_NDOF)
    return fail(c, FEM25_ERR_UNSUPPORTED,
                "dense solve: NDOF above FEM25_DENSE_MAX_NDOF (use the sparse host solver)");
  CK(cudaSetDevice(c->device), "set device");
  std::string msg;
  int r = dense_factor(c, csr128, (cudaStream_t)stream, &msg);
  return r ? fail(c, r, msg) : FEM25_OK;
}

int fem25_dense_solve_dev(fem25_ctx *h, int nrhs, int trans, double *rhs, void *stream) {
  if (!h || !rhs || nrhs <= 0 || trans < 0 || trans > 2) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  std::string msg;
  int r = dense_solve(c, nrhs, trans, rhs, (cudaStream_t)stream, &msg);
  return r ? fail(c, r, msg) : FEM25_OK;
}

int fem25_sparse_factor_dev(fem25_ctx *h, const double *csr128, void *stream) {
  if (!h || !csr128) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  std::string msg;
  int r = sparse_factor(c, csr128, (cudaStream_t)stream, &msg);
  return r ? fail(c, r, msg) : FEM25_OK;
}

int fem25_sparse_solve_dev(fem25_ctx *h, int nrhs, int trans, double *rhs, void *stream) {
  if (!h || !rhs || nrhs <= 0 || trans < 0 || trans > 2) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  std::string msg;
  int r = sparse_solve(c, nrhs, trans, rhs, (cudaStream_t)stream, &msg);
  return r ? fail(c, r, msg) : FEM25_OK;
}

int fem25_sparse_plan(const fem25_mesh *m, const fem25_graph *g, long long *out) {
  if (!m || !g || !out || !m->ieng || !m->xlocs || !m->zlocs) return FEM25_ERR_ARG;
  if (g->g.nelem != m->nelem) return FEM25_ERR_ARG;
  std::string msg;
  const int r = sparse_plan_info(m->nelem, g->g.ndof, g->g.lm.data(), m->ieng, m->xlocs,
                                 m->zlocs, out, &msg);
  if (r) std::fprintf(stderr, "fem25gpu: %s\n", msg.c_str());
  return r;
}

int fem25_sparse_info(fem25_ctx *h, long long *out) {
  if (!h || !out) return FEM25_ERR_ARG;
  sparse_info(&h->c, out);
  return FEM25_OK;
}

int fem25_addblk_dev(fem25_ctx *h, int nsrc, const float *ue, float *sol, void *stream) {
  if (!h || !ue || !sol || nsrc <= 0) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  CK(launch_addblk(c, nsrc, ue, sol, (cudaStream_t)stream), "addblk");
  return FEM25_OK;
}

// Checks shared by the gradient entry points; 0 or an error status.
static int grad_args(Ctx *c, int npairs, const double *freq, const double *py, int nsrc,
                     const double *u, const double *lam) {
  if (!freq || !py || !u || !lam || npairs <= 0 || nsrc <= 0) return FEM25_ERR_ARG;
  if (c->mesh_scalars.ldisp)
    return fail(c, FEM25_ERR_UNSUPPORTED, "gradient: dispersive media are not supported");
  if ((long long)npairs * nsrc > (1LL << 30))
    return fail(c, FEM25_ERR_ARG, "gradient: more than 2^30 (pair, source) fields");
  return 0;
}

// (omega, omega * py) of pairs [p0, p0 + np) as one launch's parameter table
static PairTable pair_table(const double *freq, const double *py, int p0, int np) {
  PairTable pt;
  for (int k = 0; k < kMaxPairs; k++) {
    const double omega = k < np ? 6.2831853071795862 * freq[p0 + k] : 0.0;
    pt.p[k] = make_double2(omega, k < np ? omega * py[p0 + k] : 0.0);
  }
  return pt;
}

// One-time set-up of the covariance gradient (allocates: not inside a capture).
static int ensure_cov(Ctx *c, cudaStream_t st) {
  if (c->d_cov) return 0;
  if (capturing(st))
    return fail(c, FEM25_ERR_ARG,
                "gradient: make one uncaptured split-precision call before capturing");
  cudaError_t e = prepare_grad_cov(c);
  if (e == cudaErrorNotSupported)
    return fail(c, FEM25_ERR_UNSUPPORTED, "gradient: split-precision path not available");
  if (e != cudaSuccess) return fail(c, FEM25_ERR_CUDA, std::string("gradient (tf32x3) set-up: ") +
                                                           cudaGetErrorString(e));
  return 0;
}

// Adds the covariances of pairs' fields into the context's accumulators, 64
// pairs per launch.
static int cov_accumulate(Ctx *c, int npairs, const double *freq, const double *py, int nsrc,
                          const double *u, const double *lam, cudaStream_t st) {
  const size_t per_pair = (size_t)nsrc * c->ndof * 2;  // doubles of one pair's fields
  for (int p0 = 0; p0 < npairs; p0 += kMaxPairs) {
    const int np = std::min(kMaxPairs, npairs - p0);
    CK(launch_grad_cov(c, pair_table(freq, py, p0, np), np, nsrc, u + p0 * per_pair,
                       lam + p0 * per_pair, st),
       "gradient (tf32x3) accumulation");
  }
  return FEM25_OK;
}

int fem25_gradient_dev(fem25_ctx *h, int npairs, const double *freq, const double *py, int nsrc,
                       const double *u, const double *lam, int prec, double *grad, void *stream) {
  if (!h || !grad) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  int r = grad_args(c, npairs, freq, py, nsrc, u, lam);
  if (r) return r;
  if (prec != FEM25_PREC_FP64 && prec != FEM25_PREC_TF32X3 && prec != FEM25_PREC_TF32X3_POINTWISE)
    return fail(c, FEM25_ERR_ARG, "gradient: unknown precision");
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(c->device), "set device");
  if (prec == FEM25_PREC_TF32X3) {
    if ((r = ensure_cov(c, st))) return r;
    if ((r = cov_accumulate(c, npairs, freq, py, nsrc, u, lam, st))) return r;
    CK(launch_grad_cov_fin(c, grad, st), "gradient (tf32x3) contraction");
    return FEM25_OK;
  }
  if (prec == FEM25_PREC_TF32X3_POINTWISE && !c->d_tc_tab) {
    if (capturing(st))
      return fail(c, FEM25_ERR_ARG,
                  "gradient: make one uncaptured split-precision call before capturing");
    cudaError_t e = prepare_grad_tc(c);
    if (e == cudaErrorNotSupported)
      return fail(c, FEM25_ERR_UNSUPPORTED, "gradient: split-precision path not available");
    CK(e, "gradient (tf32x3) set-up");
  }
  // pairs travel as kernel parameters, kMaxPairs per launch; both kernels
  // add into grad, so the chunks accumulate
  const size_t per_pair = (size_t)nsrc * c->ndof * 2;  // doubles of one pair's fields
  for (int p0 = 0; p0 < npairs; p0 += kMaxPairs) {
    const int np = std::min(kMaxPairs, npairs - p0);
    const PairTable pt = pair_table(freq, py, p0, np);
    const double *uk = u + p0 * per_pair, *lk = lam + p0 * per_pair;
    if (prec == FEM25_PREC_FP64) {
      CK(launch_grad_plain(c, pt, np, nsrc, uk, lk, grad, st), "gradient");
    } else {
      CK(launch_grad_tc(c, pt, np, nsrc, uk, lk, grad, st), "gradient (tf32x3)");
    }
  }
  return FEM25_OK;
}

int fem25_gradient_accumulate_dev(fem25_ctx *h, int npairs, const double *freq, const double *py,
                                  int nsrc, const double *u, const double *lam, void *stream) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  int r = grad_args(c, npairs, freq, py, nsrc, u, lam);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaSetDevice(c->device), "set device");
  if ((r = ensure_cov(c, st))) return r;
  return cov_accumulate(c, npairs, freq, py, nsrc, u, lam, st);
}

int fem25_gradient_finalize_dev(fem25_ctx *h, double *grad, void *stream) {
  if (!h || !grad) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (c->mesh_scalars.ldisp)
    return fail(c, FEM25_ERR_UNSUPPORTED, "gradient: dispersive media are not supported");
  CK(cudaSetDevice(c->device), "set device");
  if (!c->d_cov || !c->cov_pending) return FEM25_OK;  // nothing accumulated
  CK(launch_grad_cov_fin(c, grad, (cudaStream_t)stream), "gradient (tf32x3) contraction");
  return FEM25_OK;
}

int fem25_ref_gradient_info(fem25_ctx *h, int *nnpinv, long long *nz_fdist, int *maskg) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  if (nnpinv) *nnpinv = c->rg.nnpinv;
  if (nz_fdist) *nz_fdist = c->rg.nz;
  if (maskg) std::memcpy(maskg, c->rg.maskg.data(), sizeof(int) * c->nnpg);
  return FEM25_OK;
}

int fem25_ref_gradient_dev(fem25_ctx *h, const char *cinvtype, double vpvs, double freq,
                           double py, const float *wave, const float *adjlam, int accumulate,
                           float *gradl, void *stream) {
  if (!h || !cinvtype || !wave || !adjlam || !gradl) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  std::string ct(cinvtype, cinvtype + 2);
  int lisp;
  if (ct == "PP" || ct == "pp") lisp = 1;
  else if (ct == "SS" || ct == "ss") lisp = 0;
  else if (ct == "PS" || ct == "ps")
    return fail(c, FEM25_ERR_UNSUPPORTED, "vforce25: Error S and P derivatives not done yet");
  else return fail(c, FEM25_ERR_UNSUPPORTED, "vforce25: Error anisotropy not programmed!");
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  cudaStream_t st = (cudaStream_t)stream;
  CK(launch_ref_cfmat(c, lisp, vpvs, 6.2831853071795862 * freq, py, wave, accumulate, st), "cfmat");
  CK(launch_ref_adjflam(c, adjlam, gradl, st), "adjflam");
  return FEM25_OK;
}

int fem25_ref_met225_dev(fem25_ctx *h, const char *cinvtype, double freq, double py,
                         const float *adjlam, const float *nu, const float *alpha,
                         const float *wave, int accumulate, float *p1buf, float *p2buf,
                         void *stream) {
  if (!h || !cinvtype || !adjlam || !nu || !alpha || !wave || !p1buf || !p2buf)
    return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  std::string ct(cinvtype, cinvtype + 2);
  int lisp = 0, liss = 0;
  if (ct == "PP" || ct == "pp") lisp = 1;
  else if (ct == "SS" || ct == "ss") liss = 1;
  else if (ct == "PS" || ct == "ps") lisp = liss = 1;
  else return fail(c, FEM25_ERR_UNSUPPORTED, "met225_mod: Error anisotropy not programmed!");
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  CK(launch_ref_met225(c, lisp, liss, 6.2831853071795862 * freq, py, adjlam, nu, alpha, wave,
                       accumulate ? 1 : 0, p1buf, p2buf, (cudaStream_t)stream),
     "met225");
  return FEM25_OK;
}

int fem25_ref_cadj_nu_alpha_dev(fem25_ctx *h, const char *cinvtype, double freq, double py,
                                const float *v, const float *adjlam, const float *wave,
                                int accumulate, float *rhsbnu, float *rhsalp, float *p3,
                                void *stream) {
  if (!h || !cinvtype || !v || !adjlam || !wave || !rhsbnu || !rhsalp || !p3)
    return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  std::string ct(cinvtype, cinvtype + 2);
  int lisp = 0, liss = 0;
  if (ct == "PP" || ct == "pp") lisp = 1;
  else if (ct == "SS" || ct == "ss") liss = 1;
  else if (ct == "PS" || ct == "ps") lisp = liss = 1;
  else return fail(c, FEM25_ERR_UNSUPPORTED, "cadj_nu_alpha2: Error anisotropy not programmed!");
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  std::string msg;
  if ((r = prepare_cadj(c, &msg))) return fail(c, r, msg);
  CK(launch_ref_cadj(c, lisp, liss, 6.2831853071795862 * freq, py, v, adjlam, wave,
                     accumulate ? 1 : 0, rhsbnu, rhsalp, p3, (cudaStream_t)stream),
     "cadj_nu_alpha");
  return FEM25_OK;
}

int fem25_ref_pchadj_dev(fem25_ctx *h, int nvinv, int nrhs, const float *grns,
                         const float *fmat, float *hessb, float *jacl, void *stream) {
  if (!h || !grns || !fmat || !hessb || nrhs <= 0 || nvinv < 1 || nvinv > 2)
    return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if ((size_t)nrhs * nvinv * 8 > 200 * 1024)
    return fail(c, FEM25_ERR_UNSUPPORTED, "pchadj: more than 12 800 / nvinv right-hand sides");
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  CK(launch_ref_pchadj(c, nvinv, nrhs, grns, fmat, hessb, jacl, (cudaStream_t)stream), "pchadj");
  return FEM25_OK;
}

int fem25_ref_vforce2_dev(fem25_ctx *h, const char *cinvtype, double freq, double py,
                          const float *wave, float *fmat, void *stream) {
  if (!h || !cinvtype || !wave || !fmat) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  std::string ct(cinvtype, cinvtype + 2);
  int lisp = 0, liss = 0;
  if (ct == "PP" || ct == "pp") lisp = 1;
  else if (ct == "SS" || ct == "ss") liss = 1;
  else if (ct == "PS" || ct == "ps") lisp = liss = 1;
  else return fail(c, FEM25_ERR_ARG, "vforce25_2: CINVTYPE must be PP, SS or PS");
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  CK(launch_ref_vforce2(c, lisp, liss, 6.2831853071795862 * freq, py, wave, fmat,
                        (cudaStream_t)stream),
     "vforce25_2");
  return FEM25_OK;
}

int fem25_wtgrad_dev(fem25_ctx *h, int na35, const float *wgrad, float *grad, void *stream) {
  if (!h || !wgrad || !grad || na35 <= 0) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  CK(launch_wtgrad(na35, wgrad, grad, (cudaStream_t)stream), "wtgrad");
  return FEM25_OK;
}

// shared checks of AVGRAD / AVGRAD8: the GENGMASK tables, set up outside a capture
static int avgrad_args(Ctx *c, int nvinv, int ncasc, const void *grad, cudaStream_t st) {
  if (!grad || nvinv < 1 || nvinv > 2 || ncasc < 0) return FEM25_ERR_ARG;
  if (!c->refgrad_ready && capturing(st))
    return fail(c, FEM25_ERR_ARG,
                "avgrad: the inversion tables are built on the first call; make one uncaptured "
                "call before capturing");
  return ensure_refgrad(c);
}

int fem25_avgrad_dev(fem25_ctx *h, int nvinv, int ncasc, float *grad, void *stream) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  int r = avgrad_args(c, nvinv, ncasc, grad, (cudaStream_t)stream);
  if (r) return r;
  CK(launch_avgrad(c, nvinv, ncasc, grad, (cudaStream_t)stream), "avgrad");
  return FEM25_OK;
}

int fem25_avgrad8_dev(fem25_ctx *h, int nvinv, int ncasc, double *grad, void *stream) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  int r = avgrad_args(c, nvinv, ncasc, grad, (cudaStream_t)stream);
  if (r) return r;
  CK(launch_avgrad8(c, nvinv, ncasc, grad, (cudaStream_t)stream), "avgrad8");
  return FEM25_OK;
}

int fem25_postsolve_dev(fem25_ctx *h, int nsrc, int nrec, const int *mrdof, const double *yrec,
                        double freq, double py, double azmod, const float *recv, const float *ue,
                        float *sol, const float *obs, const float *wghts, float *est, float *rhs,
                        float *misfit, void *stream) {
  if (!h || nsrc <= 0 || nrec <= 0 || !mrdof || !yrec || !recv || !ue || !sol || !obs || !wghts ||
      !est || !rhs || !misfit)
    return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (nrec > FEM25_POSTSOLVE_MAX_REC)
    return fail(c, FEM25_ERR_ARG, "postsolve: nrec exceeds FEM25_POSTSOLVE_MAX_REC");
  {
    std::vector<int> seen;
    for (int k = 0; k < 3 * nrec; k++) {
      if (mrdof[k] < 0 || mrdof[k] > c->ndof)
        return fail(c, FEM25_ERR_ARG, "postsolve: MRDOF entry out of range");
      if (mrdof[k] > 0) seen.push_back(mrdof[k]);
    }
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
      return fail(c, FEM25_ERR_ARG, "postsolve: two receiver components share a DOF");
  }
  CK(cudaSetDevice(c->device), "set device");
  cudaStream_t st = (cudaStream_t)stream;
  // receiver tables: rebuilt only when MRDOF differs from the last call's
  if (c->post_mrdof.size() != 3 * (size_t)nrec ||
      !std::equal(c->post_mrdof.begin(), c->post_mrdof.end(), mrdof)) {
    CK(cudaStreamSynchronize(st), "synchronize");
    if (c->d_post_mrdof) cudaFree(c->d_post_mrdof);
    if (c->d_post_bits) cudaFree(c->d_post_bits);
    c->d_post_mrdof = nullptr;
    c->d_post_bits = nullptr;
    c->post_mrdof.clear();
    std::vector<uint32_t> bits(((size_t)c->ndof + 31) / 32, 0u);
    for (int k = 0; k < 3 * nrec; k++)
      if (mrdof[k] > 0) bits[(mrdof[k] - 1) >> 5] |= 1u << ((mrdof[k] - 1) & 31);
    CK(dalloc_copy(&c->d_post_mrdof, mrdof, 3 * (size_t)nrec), "postsolve");
    CK(dalloc_copy(&c->d_post_bits, bits.data(), bits.size()), "postsolve");
    c->post_mrdof.assign(mrdof, mrdof + 3 * (size_t)nrec);
  }
  const double omega = 6.2831853071795862 * freq;
  std::vector<float> trig(4 * (size_t)nrec);
  for (int ir = 0; ir < nrec; ir++) {
    float ph = (float)(omega * py * yrec[ir]);
    float ph2 = -(float)(omega * py * yrec[ir]);
    trig[4 * ir + 0] = cosf(ph);
    trig[4 * ir + 1] = sinf(ph);
    trig[4 * ir + 2] = cosf(ph2);
    trig[4 * ir + 3] = sinf(ph2);
  }
  float *d_trig = nullptr, *d_recv = nullptr, *d_obs = nullptr, *d_w = nullptr, *d_est = nullptr,
        *d_mis = nullptr;
  const size_t nr3 = 3 * (size_t)nrec, ns3 = nr3 * nsrc;
  auto run = [&]() -> int {
    CK(dalloc_copy(&d_trig, trig.data(), trig.size()), "postsolve");
    CK(dalloc_copy(&d_recv, recv, 2 * nr3), "postsolve");
    CK(dalloc_copy(&d_obs, obs, 2 * ns3), "postsolve");
    CK(dalloc_copy(&d_w, wghts, ns3), "postsolve");
    CK(cudaMalloc(&d_est, sizeof(float) * 2 * ns3), "postsolve");
    CK(cudaMalloc(&d_mis, sizeof(float) * nsrc), "postsolve");
    CK(launch_postsolve(c, nsrc, nrec, c->d_post_mrdof, c->d_post_bits, d_trig, freq, azmod, d_recv,
                        ue, sol, d_obs, d_w, d_est, rhs, d_mis, st),
       "postsolve");
    CK(cudaMemcpyAsync(est, d_est, sizeof(float) * 2 * ns3, cudaMemcpyDeviceToHost, st), "postsolve");
    CK(cudaMemcpyAsync(misfit, d_mis, sizeof(float) * nsrc, cudaMemcpyDeviceToHost, st),
       "postsolve");
    CK(cudaStreamSynchronize(st), "postsolve");
    return FEM25_OK;
  };
  int r = run();
  for (void *p : {(void *)d_trig, (void *)d_recv, (void *)d_obs, (void *)d_w, (void *)d_est,
                  (void *)d_mis})
    if (p) cudaFree(p);
  return r;
}

int fem25_asmb_peff(fem25_ctx *h, int ndof, const float *cdist, const float *ue, float *peff) {
  if (!h || !ue || !peff) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (ndof != c->ndof) return fail(c, FEM25_ERR_ARG, "asmb_peff: NDOF differs from the context");
  CK(cudaSetDevice(c->device), "set device");
  const size_t n = (size_t)c->ndof;
  if (!c->d_hvec) CK(cudaMalloc(&c->d_hvec, sizeof(float2) * 3 * n), "host-buffer scratch");
  const float2 *a_loc = c->d_cdist;
  if (cdist) {
    if (!c->d_cdist) CK(cudaMalloc(&c->d_cdist, sizeof(float2) * (size_t)c->nzero), "cdist buffer");
    CK(cudaMemcpy(c->d_cdist, cdist, sizeof(float2) * (size_t)c->nzero, cudaMemcpyHostToDevice),
       "cdist upload");
    a_loc = c->d_cdist;
  } else if (!a_loc) {
    return fail(c, FEM25_ERR_NOMESH,
                "asmb_peff: CDIST = NULL needs a fem25_asmble_driver call on this context first");
  }
  CK(cudaMemcpy(c->d_hvec, ue, sizeof(float2) * n, cudaMemcpyHostToDevice), "ue upload");
  CK(launch_peff(c, 1, (const float *)a_loc, (const float *)c->d_hvec, (float *)(c->d_hvec + n), 0),
     "peff");
  CK(cudaMemcpy(peff, c->d_hvec + n, sizeof(float2) * n, cudaMemcpyDeviceToHost), "peff copy");
  return read_err_word(c, 0);
}

int fem25_cfmat_adjgrad(fem25_ctx *h, const char *cinvtype, double vpvs, double freq, double py,
                        const float *wave, const float *adjlam, int accumulate, float *gradl) {
  if (!h || !cinvtype || !wave || !adjlam || !gradl) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  CK(cudaSetDevice(c->device), "set device");
  int r = ensure_refgrad(c);
  if (r) return r;
  const size_t n = (size_t)c->ndof;
  if (!c->d_hvec) CK(cudaMalloc(&c->d_hvec, sizeof(float2) * 3 * n), "host-buffer scratch");
  if (!c->d_hgrad)
    CK(cudaMalloc(&c->d_hgrad, sizeof(float) * (size_t)std::max(c->rg.nnpinv, 1)), "gradl buffer");
  CK(cudaMemcpy(c->d_hvec, wave, sizeof(float2) * n, cudaMemcpyHostToDevice), "wave upload");
  CK(cudaMemcpy(c->d_hvec + n, adjlam, sizeof(float2) * n, cudaMemcpyHostToDevice), "adjlam upload");
  CK(cudaMemcpy(c->d_hgrad, gradl, sizeof(float) * (size_t)c->rg.nnpinv, cudaMemcpyHostToDevice),
     "gradl upload");
  r = fem25_ref_gradient_dev(h, cinvtype, vpvs, freq, py, (const float *)c->d_hvec,
                             (const float *)(c->d_hvec + n), accumulate, c->d_hgrad, nullptr);
  if (r) return r;
  CK(cudaMemcpy(gradl, c->d_hgrad, sizeof(float) * (size_t)c->rg.nnpinv, cudaMemcpyDeviceToHost),
     "gradl copy");
  return read_err_word(c, 0);
}

int fem25_misfit_options(fem25_ctx *h, int norm, int irestp, int ibphase, float eps, float thresh,
                         float dtmax, float dtmax_obj) {
  if (!h) return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (norm < 1 || norm > 4) return fail(c, FEM25_ERR_ARG, "misfit options: NORM must be 1-4");
  if (irestp < 1 || irestp > 3) return fail(c, FEM25_ERR_ARG, "misfit options: IRESTP must be 1-3");
  if (ibphase < 0 || ibphase > 6)
    return fail(c, FEM25_ERR_ARG, "misfit options: IBPHASE must be 0-6");
  c->mopt.norm = norm;
  c->mopt.irestp = irestp;
  c->mopt.ibphase = ibphase;
  c->mopt.eps = eps;
  c->mopt.thresh = thresh;
  c->mopt.dtmax = dtmax;
  c->mopt.dtmax_obj = dtmax_obj;
  return FEM25_OK;
}

int fem25_misfit_dev(fem25_ctx *h, int nsrc, int nrec, const int *mrdof, const double *yrec,
                     double freq, double py, double azmod, const float *recv, const float *sol,
                     const float *obs, const float *wghts, float *est, float *rhs, float *misfit,
                     void *stream) {
  if (!h || nsrc <= 0 || nrec <= 0 || !mrdof || !yrec || !recv || !sol || !obs || !wghts || !est ||
      !rhs || !misfit)
    return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  {
    std::vector<int> seen;
    for (int k = 0; k < 3 * nrec; k++) {
      if (mrdof[k] < 0 || mrdof[k] > c->ndof)
        return fail(c, FEM25_ERR_ARG, "misfit: MRDOF entry out of range");
      if (mrdof[k] > 0) seen.push_back(mrdof[k]);
    }
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end())
      return fail(c, FEM25_ERR_ARG, "misfit: two receiver components share a DOF");
  }
  CK(cudaSetDevice(c->device), "set device");
  cudaStream_t st = (cudaStream_t)stream;
  const double omega = 6.2831853071795862 * freq;
  std::vector<float> trig(4 * (size_t)nrec);
  for (int ir = 0; ir < nrec; ir++) {
    float ph = (float)(omega * py * yrec[ir]);
    float ph2 = -(float)(omega * py * yrec[ir]);
    trig[4 * ir + 0] = cosf(ph);
    trig[4 * ir + 1] = sinf(ph);
    trig[4 * ir + 2] = cosf(ph2);
    trig[4 * ir + 3] = sinf(ph2);
  }
  int *d_mrdof = nullptr;
  float *d_trig = nullptr, *d_recv = nullptr, *d_obs = nullptr, *d_w = nullptr, *d_est = nullptr,
        *d_mis = nullptr;
  const size_t nr3 = 3 * (size_t)nrec, ns3 = nr3 * nsrc;
  int r = FEM25_OK;
  auto run = [&]() -> int {
    CK(dalloc_copy(&d_mrdof, mrdof, nr3), "misfit");
    CK(dalloc_copy(&d_trig, trig.data(), trig.size()), "misfit");
    CK(dalloc_copy(&d_recv, recv, 2 * nr3), "misfit");
    CK(dalloc_copy(&d_obs, obs, 2 * ns3), "misfit");
    CK(dalloc_copy(&d_w, wghts, ns3), "misfit");
    CK(cudaMalloc(&d_est, sizeof(float) * 2 * ns3), "misfit");
    CK(cudaMalloc(&d_mis, sizeof(float) * nsrc), "misfit");
    CK(launch_misfit(c, nsrc, nrec, d_mrdof, d_trig, freq, py, azmod, d_recv, sol, d_obs, d_w,
                     d_est, rhs, d_mis, st),
       "misfit");
    CK(cudaMemcpyAsync(est, d_est, sizeof(float) * 2 * ns3, cudaMemcpyDeviceToHost, st), "misfit");
    CK(cudaMemcpyAsync(misfit, d_mis, sizeof(float) * nsrc, cudaMemcpyDeviceToHost, st), "misfit");
    CK(cudaStreamSynchronize(st), "misfit");
    return FEM25_OK;
  };
  r = run();
  for (void *p : {(void *)d_mrdof, (void *)d_trig, (void *)d_recv, (void *)d_obs, (void *)d_w,
                  (void *)d_est, (void *)d_mis})
    if (p) cudaFree(p);
  return r;
}

}  // extern "C"
