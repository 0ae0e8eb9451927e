// Device context of libfem25gpu and the kernel entry points shared between
// translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include <string>
#include <vector>

#include "fem25_internal.h"

namespace fem25 {

// Quadrature tables on the device (built once by build_tables()).
struct DevTables {
  double *xigll;  // [13]
  double *wts;    // [13]
  double *shl;    // [169][25][3]  SHL(3,NEN,NINT,NINT)
  double *sf;     // [169][4]
  double *dsf;    // [169][2][4]
};

// Per-(omega, cftype) PML parameters resolved on the host (asmble.f90:78-88).
struct PmlParams {
  double omega, rcoeff, dmax, kappa, fcent, xwidth, zwidth;
};

// Arguments of the element kernels that read the mesh.
struct MeshView {
  int nelem, nnpg;
  const int4 *ieng;        // 1-based anchors, one int4 per element
  const char *cdomain;
  const double *x, *z, *xd, *zd, *lam, *mu, *rho;
  const double *qp, *qs;   // quality factors (dispersive media only, else null)
};

// One (omega, py) system of a batch, pre-digested for the streaming kernel.
struct SysParam {
  double w2;     // omega^2
  double wpy;    // omega * py
  int pml_slot;  // index of the PML delta of this system's (omega, cftype)
  int pad;
};

constexpr int kMaxPass = 16;  // systems per streaming launch

// The systems of one streaming launch, passed by value as a kernel parameter.
struct SysTable {
  SysParam s[kMaxPass];
};

constexpr int kMaxBatch = 1024;  // systems per launch of the large-batch streaming kernel

// The systems of one large-batch streaming launch (24 KB kernel parameter).
struct SysTableBig {
  SysParam s[kMaxBatch];
};

constexpr int kMaxPairs = 64;  // (omega, py) pairs per gradient launch

// (omega, omega * py) of the pairs of one gradient launch, passed by value.
struct PairTable {
  double2 p[kMaxPairs];
};

// Options of the misfit / adjoint source (the reference's INV_INFO fields
// NORM, IRESTP, IBPHASE, the thresholds of COBJ4 and the DTMAX phase-jump
// tests), and the per-call values the kernel needs.
struct MisfitOpts {
  int norm, irestp, ibphase;
  float eps, thresh;       // COBJ4's EPS = EPSS * CRESMN, THRESH = THRESHS * CRESMN
  float dtmax, dtmax_obj;  // BPRESID4's and COBJ4's DTMAX (0 = off)
  double freq;             // FREQ of the call
  float2 hfact;            // HDIFFER(IBPHASE, FREQ) of the call
};

struct DenseLU;   // dense LU of the small-mesh direct solve (dense_solve.cu)
struct SparseLU;  // multifrontal LU of the sparse direct solve (sparse_solve.cu)

struct Ctx {
  int device = 0;
  std::string err;
  fem25_mesh mesh_scalars{};   // scalars only (pointers not kept)
  int nelem = 0, nnpg = 0, ndof = 0;
  long long nzero = 0;
  Tables tab;
  DevTables dt{};
  MeshView mv{};
  // device mesh arrays
  int4 *d_ieng = nullptr;
  char *d_cdomain = nullptr;
  double *d_x = nullptr, *d_z = nullptr, *d_xd = nullptr, *d_zd = nullptr;
  double *d_lam = nullptr, *d_mu = nullptr, *d_rho = nullptr;
  double *d_qp = nullptr, *d_qs = nullptr;  // dispersive media
  std::vector<char> h_cdomain, h_cnnpg;
  std::vector<double> h_x, h_z;
  std::vector<int> h_ieng, h_lm, h_irptr;
  // graph
  int *d_lm = nullptr, *d_irptr = nullptr, *d_jcptr = nullptr;
  char *d_cnp = nullptr;
  // plain path: element matrices and the nonzero -> contributions gather map
  double2 *d_elemmat = nullptr;  // [nelem][625][9]
  int *d_gptr = nullptr;         // [nzero+1]
  int *d_glist = nullptr;        // contribution ids, element order per nonzero
  long long ncontrib = 0;
  int *d_err = nullptr;          // device error word
  // batched path
  BlockCSR bcsr;
  long long *d_brptr = nullptr;
  int *d_brow = nullptr;
  double *d_basis = nullptr;     // [12][nblocks]
  double *d_prim = nullptr;      // [nzero] K0/K1 basis value of every CSR entry
  unsigned *d_desc = nullptr;    // [nzero] block << 4 | i << 2 | j
  int stream_variant = -1;       // loop order of the streaming kernel (-1: not tuned yet)
  int grad_tile = -1;            // source tile of the FP64 gradient (-1: not tuned yet)
  double *d_ebasis = nullptr;    // [nelem][625][12] scratch
  int *d_bgptr = nullptr, *d_bglist = nullptr;  // block -> (element node pair) ids
  bool basis_valid = false;
  // PML part of the batched path
  int npml_elem = 0;
  int *d_pml_elems = nullptr;    // element ids of 'A' elements
  long long npml_blocks = 0;
  int *d_pml_idx = nullptr;      // [nblocks] -> PML block index or -1
  int *d_pgptr = nullptr, *d_pglist = nullptr;  // PML block -> (pml elem, ab) ids
  double2 *d_pml_emat = nullptr; // [npml_elem][625][9] scratch (one omega)
  double2 *d_pml_delta = nullptr; // [nslots_pml][npml_blocks][9][2] (CE0, CE1)
  int pml_delta_cap = 0;
  // reference-compatible gradient
  bool refgrad_ready = false;
  RefGradSetup rg;
  int *d_jcsc = nullptr, *d_icsc = nullptr, *d_rg_anchor = nullptr, *d_mconn = nullptr;
  int *d_maskg = nullptr;          // MASKG(NNPG) of GENGMASK
  void *d_avg_work = nullptr;      // AVGRAD / AVGRAD8 workspace (2 x NNPINV doubles)
  double *d_elem_wts = nullptr;
  float2 *d_fmat = nullptr;
  // CADJ_NU_ALPHA: (anchor column, connected element) pairs in the reference's
  // loop order, each DOF's (pair, local DOF) list, and the weighted blocks
  int cadj_npairs = -1;
  int *d_cadj_col0 = nullptr;  // [nnpinv + 1] first pair of each column
  int *d_cadj_pair_col = nullptr, *d_cadj_pair_elem = nullptr;
  int *d_cadj_dptr = nullptr, *d_cadj_dent = nullptr;
  float2 *d_cadj_w = nullptr;
  size_t cadj_w_cap = 0;
  // gradient
  int *d_nonpml = nullptr;       // ids of the elements outside the PML
  int n_nonpml = 0;
  unsigned char *d_tc_tab = nullptr;  // SHL tables of the tensor-core gradient (tf32 hi/lo)
  // covariance gradient: per element outside the PML, 15 FP64 blocks of
  // 25 x 25 field covariances; pending = holds sums not yet contracted
  double *d_cov = nullptr;
  bool cov_pending = false;
  // its gather plan (TMA boxes per element) and the tensor-map encoder
  int2 *d_cov_ops = nullptr;
  int *d_cov_opptr = nullptr, *d_cov_tx = nullptr;
  uint32_t *d_cov_node = nullptr;
  void *tmap_encode = nullptr;
  int *d_cov_exps = nullptr;  // per launch: the pairs' field-scale exponents
  // cached COMPLEX*8 device buffer of fem25_asmble_driver, and its pipeline:
  // element chunk k = [drv_elem[k], drv_elem[k+1]) completes the CSR rows
  // [drv_row[k], drv_row[k+1]), whose values are gathered and copied to the
  // host on copy_st while the next chunk computes
  float2 *d_cdist = nullptr;
  std::vector<int> drv_elem, drv_row;
  cudaStream_t copy_st = nullptr;
  std::vector<cudaEvent_t> drv_ev;
  DenseLU *dense = nullptr;
  SparseLU *sparse = nullptr;
  // fem25_assemble_dev with the FMA build of the element kernels
  bool plain_fma = false;
  // bounded waits of the tensor-core gradient kernels: limit in SM clocks
  // (0: the default, about half a second) and the time-out test hook
  long long wait_limit = 0;
  int wait_inject = 0;
  // receiver tables of the fused post-solve pass, kept while MRDOF repeats:
  // the receiver DOFs as a bitmap (one bit per DOF) and MRDOF itself
  std::vector<int> post_mrdof;
  int *d_post_mrdof = nullptr;
  uint32_t *d_post_bits = nullptr;
  // device scratch of the host-buffer drop-ins (fem25_asmb_peff,
  // fem25_cfmat_adjgrad): 3 COMPLEX*8 [NDOF] vectors and GRADL
  float2 *d_hvec = nullptr;
  float *d_hgrad = nullptr;
  // misfit options (fem25_misfit_options); the defaults of the reference
  MisfitOpts mopt{2, 3, 0, 0.0f, 0.0f, 0.0f, 0.0f, 0.0, {1.0f, 0.0f}};
  // optional CUDA-event timing of the dominant kernels
  bool prof = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

// kernels / launchers (defined in the .cu files)
cudaError_t launch_elem_plain(Ctx *c, char cftype, double freq, double py, int e0, int e1,
                              cudaStream_t st);
// the same element kernels compiled with FMA contraction (fem25_plain_fma)
cudaError_t launch_elem_plain_fma(Ctx *c, char cftype, double freq, double py, int e0, int e1,
                                  cudaStream_t st);
cudaError_t launch_gather_plain(Ctx *c, double *csr128, float *csr64, long long nz0,
                                long long nz1, cudaStream_t st);
cudaError_t build_gather_map(Ctx *c, cudaStream_t st);
cudaError_t check_jacobians(Ctx *c, cudaStream_t st);
cudaError_t build_batch_structures(Ctx *c, cudaStream_t st);
cudaError_t build_basis(Ctx *c, cudaStream_t st);
cudaError_t build_pml_delta(Ctx *c, const PmlParams &pp, int slot, cudaStream_t st);
cudaError_t launch_stream_batch(Ctx *c, int n, const SysParam *hsys, double *ring_base,
                                long long slot_stride, int nslots, cudaStream_t st);
cudaError_t launch_peff(Ctx *c, int nsrc, const float *a_loc, const float *ue, float *peff,
                        cudaStream_t st);
cudaError_t launch_addblk(Ctx *c, int nsrc, const float *u0, float *sol, cudaStream_t st);
int dense_factor(Ctx *c, const double *csr128, cudaStream_t st, std::string *msg);
int dense_solve(Ctx *c, int nrhs, int trans, double *rhs, cudaStream_t st, std::string *msg);
void free_dense(Ctx *c);
int sparse_factor(Ctx *c, const double *csr128, cudaStream_t st, std::string *msg);
int sparse_solve(Ctx *c, int nrhs, int trans, double *rhs, cudaStream_t st, std::string *msg);
void sparse_info(const Ctx *c, long long *out);
int sparse_plan_info(int nelem, int ndof, const int *lm, const int *ieng, const double *x,
                     const double *z, long long *out, std::string *msg);
void free_sparse(Ctx *c);
cudaError_t launch_grad_plain(Ctx *c, const PairTable &pt, int npairs, int nsrc, const double *u,
                              const double *lam, double *grad, cudaStream_t st);
cudaError_t prepare_grad_tc(Ctx *c);
cudaError_t launch_grad_tc(Ctx *c, const PairTable &pt, int npairs, int nsrc, const double *u,
                           const double *lam, double *grad, cudaStream_t st);
cudaError_t prepare_grad_cov(Ctx *c);
cudaError_t launch_grad_cov(Ctx *c, const PairTable &pt, int npairs, int nsrc, const double *u,
                            const double *lam, cudaStream_t st);
cudaError_t launch_grad_cov_fin(Ctx *c, double *grad, cudaStream_t st);
cudaError_t launch_ref_cfmat(Ctx *c, int lisp, double vpvs, double omega, double py,
                             const float *wave, int accumulate, cudaStream_t st);
cudaError_t launch_ref_adjflam(Ctx *c, const float *adjlam, float *gradl, cudaStream_t st);
cudaError_t launch_wtgrad(int na35, const float *wgrad, float *grad, cudaStream_t st);
cudaError_t launch_avgrad(Ctx *c, int nvinv, int ncasc, float *grad, cudaStream_t st);
cudaError_t launch_avgrad8(Ctx *c, int nvinv, int ncasc, double *grad, cudaStream_t st);
cudaError_t launch_ref_pchadj(Ctx *c, int nvinv, int nrhs, const float *grns, const float *fmat,
                              float *hessb, float *jacl, cudaStream_t st);
int prepare_cadj(Ctx *c, std::string *msg);
cudaError_t launch_ref_cadj(Ctx *c, int lisp, int liss, double omega, double py, const float *v,
                            const float *adjlam, const float *wave, int accumulate, float *rhsbnu,
                            float *rhsalp, float *p3, cudaStream_t st);
cudaError_t launch_ref_met225(Ctx *c, int lisp, int liss, double omega, double py,
                              const float *adjlam, const float *nu, const float *alpha,
                              const float *wave, int accumulate, float *p1buf, float *p2buf,
                              cudaStream_t st);
cudaError_t launch_ref_vforce2(Ctx *c, int lisp, int liss, double omega, double py,
                               const float *wave, float *fmat, cudaStream_t st);
cudaError_t launch_misfit(Ctx *c, int nsrc, int nrec, const int *d_mrdof, const float *d_trig,
                          double freq, double py, double azmod, const float *d_recv,
                          const float *sol, const float *d_obs, const float *d_wghts,
                          float *d_est, float *rhs, float *d_misfit, cudaStream_t st);

cudaError_t launch_misfit_part(Ctx *c, int nsrc, int nrec, const int *d_mrdof, const float *d_trig,
                               double freq, double azmod, const float *d_recv, const float *sol,
                               const float *d_obs, const float *d_wghts, float *d_est, float *rhs,
                               float *d_part, float *d_misfit, cudaStream_t st);

cudaError_t launch_postsolve(Ctx *c, int nsrc, int nrec, const int *d_mrdof, const uint32_t *d_bits,
                             const float *d_trig, double freq, double azmod, const float *d_recv,
                             const float *ue, float *sol, const float *d_obs, const float *d_wghts,
                             float *d_est, float *rhs, float *d_misfit, cudaStream_t st);

PmlParams pml_params(const Ctx *c, char cftype, double freq);

}  // namespace fem25
