/*
 * fem25gpu.h -- C ABI of the B200 (sm_100a) library for the fem25 hot path:
 * 2.5D spectral-element operator assembly into CSR per (omega, py), the
 * Bielak effective force, the forward misfit / adjoint source and the adjoint
 * gradient.
 *
 * Conventions kept from the reference Fortran (bakerb845/fem25) so that its
 * drivers can bind these entry points through ISO_C_BINDING unchanged:
 *   - every entry point returns an int status, 0 = OK (the reference's IERR);
 *     nothing aborts or exits; the last error text is kept per context;
 *   - index arrays hold Fortran 1-based values (IENG, LM, IRPTR, JCPTR ...)
 *     and two-dimensional arrays keep their Fortran column-major layout;
 *   - buffers belong to the caller; complex values are interleaved (re, im).
 * A context is not re-entrant; several contexts may run on separate streams.
 * `stream` arguments are cudaStream_t values passed as void* (NULL = default).
 */
#ifndef FEM25GPU_H
#define FEM25GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define FEM25_OK 0
#define FEM25_ERR_ARG 1          /* bad argument or size mismatch            */
#define FEM25_ERR_JACOBIAN 2     /* undefined/negative Jacobian, cjac.f:115-125 */
#define FEM25_ERR_PATTERN 3      /* (row,col) not in CSR, asmble.f90:296-300  */
#define FEM25_ERR_CUDA 4         /* CUDA runtime error                         */
#define FEM25_ERR_ALLOC 5        /* device or host allocation failed           */
#define FEM25_ERR_GRAPH 6        /* mesh graph construction failed            */
#define FEM25_ERR_UNSUPPORTED 7  /* anisotropy, dispersion, CINVTYPE 'PS' ...  */
#define FEM25_ERR_NOMESH 8       /* context lacks a table the call needs      */

/* Mesh as read by RDMESHBK (mesh_utils.f:982-1165), fields of MESH_INFO
 * (fwd_struc.h:10-141).  Isotropic (INPTYP 1/2), NGNOD = 4 anchors. */
typedef struct fem25_mesh {
    int nelem;               /* NELEM                                        */
    int nnpg;                /* NNPG, anchor nodes                           */
    int nord;                /* NORD, polynomial order (NLXI = NORD+1)       */
    int ldisp;               /* LDISP: 1 = dispersive media (qp, qs, freq0)   */
    const int *ieng;         /* IENG(4,NELEM), 1-based                        */
    const char *cdomain;     /* CDOMAIN(NELEM): 'I','E','A'                   */
    const char *cnnpg;       /* CNNPG(NNPG): CHARACTER(2), 2 bytes per anchor */
    const double *xlocs, *zlocs;  /* anchor coordinates (m)                   */
    const double *xd, *zd;   /* anchor depth into the PML (m)                 */
    const double *ecoeff;    /* ECOEFF(NNPG,2): lambda then mu (Pa)           */
    const double *dens;      /* DENS(NNPG) (kg/m^3)                           */
    double xwidth, zwidth;   /* PML widths (max XD, max ZD)                   */
    double rcoeff_srf, dmax_srf, kappa_srf, fcent_srf;  /* CFTYPE 'S'         */
    double rcoeff_bdy, dmax_bdy, kappa_bdy, fcent_bdy;  /* CFTYPE 'B'         */
    /* dispersive media (read only when ldisp = 1; RDMESHBK IDISP > 0,
     * mesh_utils.f:1082-1133): the assembly uses the complex velocities of
     * VCMPLX (haskattn.f:602-646) in KMDAMP / CMDAMP (estiff25.f:511-961) */
    const double *qp, *qs;   /* QP(NNPG), QS(NNPG) quality factors; 9999 = none */
    double freq0;            /* FREQ0 reference frequency (Hz); 0 = none      */
} fem25_mesh;

typedef struct fem25_graph fem25_graph;  /* host graph (opaque)            */
typedef struct fem25_ctx fem25_ctx;      /* device context (opaque)        */

/* ---- mesh graph: replaces GEN_GRAPH25 (graph25_driver.f90:2-72) ----------
 * GENIEN -> GENID -> GENLM -> CONNECT -> GENCRS_QUICK -> CNMESH with the
 * reference's node de-duplication tolerance (1e-8), Dirichlet rules on 'A'
 * elements, element-order DOF numbering and sorted, de-duplicated columns. */
int fem25_graph_build(const fem25_mesh *m, fem25_graph **out);
int fem25_graph_info(const fem25_graph *g, int *nnp, int *ndof, long long *nzero);
/* any pointer may be NULL; sizes: ien[NEN*NELEM], lm[3*NEN*NELEM],
 * irptr[NDOF+1], jcptr[NZERO], cnp[NDOF] */
int fem25_graph_copy(const fem25_graph *g, int *ien, int *lm, int *irptr, int *jcptr, char *cnp);
void fem25_graph_free(fem25_graph *g);

/* A cache of the graph: fem25_graph_save writes IEN, LM, IRPTR, JCPTR and CNP
 * with a fingerprint of the mesh (IENG, CDOMAIN, CNNPG, XLOCS, ZLOCS);
 * fem25_graph_load reads them back for the same mesh, so later runs skip the
 * graph build, and returns FEM25_ERR_GRAPH for a file made from another
 * mesh or a truncated one. */
int fem25_graph_save(const fem25_graph *g, const fem25_mesh *m, const char *path);
int fem25_graph_load(const fem25_mesh *m, const char *path, fem25_graph **out);

/* ---- mesh files: replaces RDMESHBK (mesh_utils.f:982-1165) ----------------
 * Reads PROJNM.nodes (NELEM; CDOMAIN, IENG(1:4) per element) and PROJNM.mesh
 * (NNPG, INPTYP, NORD, IITYPE, IDISP; XLATMIN, XLONMIN, XLATMAX, XLONMAX;
 * CNNPG, X, Z, XD, ZD, VARS(1:NCOEFF), DENS [, QP, QS] per anchor) with
 * Fortran list-directed rules.  INPTYP 1 converts (Vp, Vs) to (lambda, mu)
 * as the reference does; XWIDTH / ZWIDTH are the largest XD / ZD.  Returns
 * FEM25_ERR_ARG for a missing file or a premature end, and
 * FEM25_ERR_UNSUPPORTED (with the file still returned) for anisotropic
 * models (INPTYP > 2) or IITYPE other than 1 (GLL nodes), which this library
 * does not assemble.  fem25_mesh_file_get points a fem25_mesh at the file's
 * arrays (valid until fem25_mesh_file_free) and leaves the PML parameters
 * (RCOEFF, DMAX, KAPPA, FCENT: the reference's parameter file) and FREQ0 at
 * zero for the caller to set; ints (nullable): INPTYP, IITYPE, IDISP,
 * NELEME, NABS; reals (nullable): XLATMIN, XLONMIN, XLATMAX, XLONMAX. */
typedef struct fem25_mesh_file fem25_mesh_file;
int fem25_read_mesh(const char *projnm, fem25_mesh_file **out);
int fem25_mesh_file_get(const fem25_mesh_file *f, fem25_mesh *m, int *ints, double *reals);
void fem25_mesh_file_free(fem25_mesh_file *f);
/* FAZMOD (mesh_utils.f:1166-1212) with VINCENTY (distaz.f:141-298): model
 * azimuth in degrees from the Bielak/absorbing corners (XLATMIN, XLONMIN) ->
 * (XLATMAX, XLONMAX) on WGS-84; the AZMOD that fem25_misfit_dev takes.
 * FEM25_ERR_ARG when the iteration does not converge (near-antipodal corners,
 * where the reference falls back to a routine outside its repository). */
int fem25_fazmod(double xlatmin, double xlonmin, double xlatmax, double xlonmax, double *azmod);

/* ---- context --------------------------------------------------------------
 * Copies mesh, model and graph (LM, IRPTR, JCPTR, CNP as GEN_GRAPH25 leaves
 * them in MESH_INFO) to `device` and builds the element-to-nonzero map.
 * Returns FEM25_ERR_JACOBIAN if an element has a non-positive Jacobian and
 * FEM25_ERR_PATTERN if an element entry has no CSR slot. */
int fem25_create(const fem25_mesh *m, int ndof, long long nzero, const int *lm,
                 const int *irptr, const int *jcptr, const char *cnp, int device,
                 fem25_ctx **out);
void fem25_destroy(fem25_ctx *ctx);
int fem25_last_error(const fem25_ctx *ctx, char *buf, int n);
int fem25_sizes(const fem25_ctx *ctx, int *ndof, long long *nzero, long long *nblocks);

/* New model per outer iteration (UPDMOD, gengmask.f90:657): ECOEFF(NNPG,2)
 * and DENS(NNPG), host pointers.  Invalidates the batched-assembly basis. */
int fem25_update_model(fem25_ctx *ctx, const double *ecoeff, const double *dens);

/* ---- assembly -------------------------------------------------------------
 * Drop-in for ASMBLE_DRIVER(NZLOC,CFTYPE,FREQ,PY,MSH,CDIST,IERR)
 * (asmble.f90:1-2): fills the host COMPLEX*8 CDIST(NZLOC) (mid%A_LOC order)
 * with the reference's own arithmetic (FP64 element matrices, FP32
 * accumulation in element order).  Single process: NZLOC = NZERO. */
int fem25_asmble_driver(fem25_ctx *ctx, int nzloc, char cftype, double freq, double py,
                        float *cdist);

/* Plain per-(omega,py) FP64 assembly on device buffers.  csr128: complex128
 * values summed in FP64 in element order (NZERO x 2 doubles); csr64: the
 * reference's COMPLEX*8 accumulation.  Either may be NULL. */
int fem25_assemble_dev(fem25_ctx *ctx, char cftype, double freq, double py, double *csr128,
                       float *csr64, void *stream);

/* Benchmark option of fem25_assemble_dev (no counterpart in the reference):
 * enable = 1 computes the element matrices with the same kernels compiled
 * with fused multiply-adds, so the CSR is no longer bit-identical to the
 * reference arithmetic (it stays within about 1e-15 of it per row);
 * enable = 0 (the default) restores the separately rounded operations.
 * fem25_asmble_driver always uses the reference arithmetic. */
int fem25_plain_fma(fem25_ctx *ctx, int enable);

/* Batched assembly of n systems (cftype[k], freq[k], py[k]) into complex128
 * device slots: system k goes to ring_base + (k % nslots) * slot_stride
 * doubles (slot_stride even and >= 2*NZERO).  Uses the per-mesh affine basis
 * (built on first use) and streaming launches of up to min(16, nslots)
 * systems (min(1024, nslots) with the large-ring variants).  Slots
 * that start on 128-byte boundaries (ring_base 128-byte aligned, slot_stride
 * a multiple of 16) are written faster.  The first call builds the basis and
 * times the streaming variants (synchronously); later calls only enqueue
 * kernels, with the system parameters passed by value, and may be recorded
 * into a CUDA graph. */
int fem25_assemble_batch_dev(fem25_ctx *ctx, int n, const char *cftype, const double *freq,
                             const double *py, double *ring_base, long long slot_stride,
                             int nslots, void *stream);

/* ---- Bielak effective force ------------------------------------------------
 * Drop-in for ASMB_PEFF (asmble.f90:318-377) for nsrc background fields at
 * once: ue, peff are COMPLEX*8 [nsrc][NDOF]; a_loc is the COMPLEX*8 CSR.
 * Device pointers. */
int fem25_peff_dev(fem25_ctx *ctx, int nsrc, const float *a_loc, const float *ue, float *peff,
                   void *stream);

/* Host-buffer drop-in for ASMB_PEFF(MASTER, MYCOMM, NDOF, NDOFL, NZLOC, CNP,
 * MYDOFS, IRPTR_LOC, JCPTR_LOC, CDIST, UE, PEFF) (asmble.f90:318-319;
 * callers bielak25.f90:536, funcgradh.f90:233): ue and peff are host
 * COMPLEX*8 [NDOF] arrays; cdist is the host COMPLEX*8 CDIST(NZLOC) to
 * upload, or NULL to use the CDIST of the last fem25_asmble_driver call on
 * this context, which is still on the device (the reference calls ASMB_PEFF
 * right after ASMBLE_DRIVER for the same system).  Synchronous. */
int fem25_asmb_peff(fem25_ctx *ctx, int ndof, const float *cdist, const float *ue, float *peff);

/* ---- direct solve on the GPU (small meshes) ---------------------------------
 * Stands in for the host MUMPS factor / solve hop (forward solve
 * bielak25.f90:443-446, 545-551; transpose adjoint solve adjgrad.f90:327-341)
 * when NDOF <= FEM25_DENSE_MAX_NDOF: fem25_dense_factor_dev expands the
 * complex128 CSR (the output of fem25_assemble_dev / _batch_dev, device) into
 * a dense matrix (NDOF^2 x 16 bytes of device memory, kept by the context)
 * and factors it by LU with partial pivoting; it synchronises the stream and
 * returns FEM25_ERR_ARG for an exactly singular pivot.  fem25_dense_solve_dev
 * then solves op(A) X = B in place for nrhs complex128 columns [nrhs][NDOF]
 * on the device; trans = 0: A, 1: A^T (MUMPS ICNTL(9) != 1), 2: A^H. */
#define FEM25_DENSE_MAX_NDOF 40000
int fem25_dense_factor_dev(fem25_ctx *ctx, const double *csr128, void *stream);
int fem25_dense_solve_dev(fem25_ctx *ctx, int nrhs, int trans, double *rhs, void *stream);

/* ---- sparse direct solve on the GPU (any mesh size) -------------------------
 * The same hop as fem25_dense_*, for meshes of any size (replaces the host
 * MUMPS factor / solve, bielak25.f90:443-446, 545-551, and the transpose
 * adjoint solve, adjgrad.f90:327-341): multifrontal LU of the complex128 CSR
 * (device) with a nested-dissection ordering of the elements, partial
 * pivoting within each front's fully summed rows, the factors kept by the
 * context (fem25_sparse_info reports their size).  The first call analyses
 * the mesh (host, seconds for millions of DOFs) and allocates; every call
 * synchronises the stream and returns FEM25_ERR_ARG for a zero pivot.
 * fem25_sparse_solve_dev solves op(A) X = B in place for nrhs complex128
 * columns [nrhs][NDOF] on the device; trans = 0: A, 1: A^T, 2: A^H.
 * fem25_sparse_info fills out[7] = {fronts, levels, factor bytes, work-buffer
 * bytes, largest front's fully summed DOFs, largest front's order, real
 * flops of one factorisation (8 per complex multiply-add)}; zeros before the
 * first factorisation. */
int fem25_sparse_factor_dev(fem25_ctx *ctx, const double *csr128, void *stream);
int fem25_sparse_solve_dev(fem25_ctx *ctx, int nrhs, int trans, double *rhs, void *stream);
int fem25_sparse_info(fem25_ctx *ctx, long long *out);
/* The nested dissection that fem25_sparse_factor_dev would use for a mesh and
 * its graph (fem25_graph_build), computed on the host without a device or a
 * context: out[7] as fem25_sparse_info.  For planning memory (the factor
 * store and the two work buffers) before a context exists. */
int fem25_sparse_plan(const fem25_mesh *mesh, const fem25_graph *graph, long long *out);

/* Drop-in for ADDBLK (bielak_utils.f:1116-1125; callers funcgradh.f90:248,
 * srcrec.f90:694, fgh_window.f90:437, qpmfree.f90:378): after the solve, the
 * background field is added back on the exterior ('E') DOFs,
 * sol(i) += ue(i) in COMPLEX*8, for nsrc solutions at once; ue and sol are
 * COMPLEX*8 [nsrc][NDOF] device arrays, sol updated in place. */
int fem25_addblk_dev(fem25_ctx *ctx, int nsrc, const float *ue, float *sol, void *stream);

/* ---- adjoint gradient -------------------------------------------------------
 * Exact gradient of the misfit with respect to the anchor-node lambda, mu and
 * rho:  grad[m*NNPG + p] += sum_s Re( lam_s^H (dA/dm_p) u_s )
 * for m = lambda, mu, rho, summed over the n (omega, py) pairs; fields are
 * complex128 device arrays [pair][src][NDOF]; grad is FP64 on the device.
 * Replaces the per-source CFMAT_DIST + ADJGRAD sums (hessloc.f90:1-133,
 * adjgrad.f90:1-145) and the MPI_REDUCE of GRADL (funcgradh.f90:428) for an
 * exact (not Vp/Vs-masked) parameterisation.
 * Elements of domain 'A' (PML) do not contribute.
 * prec:
 *   FEM25_PREC_FP64             plain FP64 kernels, per (pair, source) at the
 *                               169 quadrature points;
 *   FEM25_PREC_TF32X3           split-precision tensor cores (3xTF32, FP32
 *                               accumulation in TMEM, FP64 across pairs):
 *                               per element the weighted covariances
 *                               sum conj(lam) u^T of the nodal fields are
 *                               accumulated over all pairs and sources, then
 *                               contracted once in FP64.  Equivalent to
 *                               fem25_gradient_accumulate_dev followed by
 *                               fem25_gradient_finalize_dev, so it also adds
 *                               any accumulation still pending on the context.
 *                               Within 1e-6 of FP64 per parameter on smooth
 *                               fields; on solved point-source fields mu and
 *                               rho stay within 1e-6 while lambda, whose
 *                               divergence terms cancel for shear-dominated
 *                               fields, can reach a few 1e-6;
 *   FEM25_PREC_TF32X3_POINTWISE split-precision tensor cores interpolating
 *                               both fields at the 169 points per (pair,
 *                               source), no accumulator memory; within 1e-6
 *                               of FP64 for lambda, mu and rho on smooth and
 *                               solved fields; faster for one-shot calls
 *                               with few (pair, source) fields, as the
 *                               covariance form's contraction is a fixed
 *                               cost per call (about 40 fields on a
 *                               48 000-element mesh break even).
 * Pairs are passed to the kernels by value, 64 per launch; the call only
 * enqueues work and may be recorded into a CUDA graph once the first
 * split-precision call of that kind on the context (which allocates or
 * uploads its tables) has returned. */
#define FEM25_PREC_FP64 0
#define FEM25_PREC_TF32X3 1
#define FEM25_PREC_TF32X3_POINTWISE 2
int fem25_gradient_dev(fem25_ctx *ctx, int npairs, const double *freq, const double *py,
                       int nsrc, const double *u, const double *lam, int prec, double *grad,
                       void *stream);

/* Split form of the FEM25_PREC_TF32X3 gradient for inversion loops that
 * solve one pair at a time (funcgradh.f90:191-420: every frequency's forward
 * and adjoint fields add into GRADL before one reduction).
 * fem25_gradient_accumulate_dev adds the covariances of npairs pairs'
 * fields (same arguments as fem25_gradient_dev) into the context's
 * accumulators: 15 x 625 doubles per element outside the PML (75 KB each),
 * allocated by the first call, which must not be inside a stream capture.
 * fem25_gradient_finalize_dev contracts everything accumulated since the
 * last finalize into grad (+=) and empties the accumulators; with nothing
 * accumulated it leaves grad unchanged.  The first accumulation after a
 * finalize overwrites the accumulators instead of adding, a choice made
 * when the call is made: a CUDA graph should record accumulate calls
 * together with the finalize that consumes them. */
int fem25_gradient_accumulate_dev(fem25_ctx *ctx, int npairs, const double *freq,
                                  const double *py, int nsrc, const double *u, const double *lam,
                                  void *stream);
int fem25_gradient_finalize_dev(fem25_ctx *ctx, double *grad, void *stream);

/* Reference-compatible gradient (CFMAT_DIST hessloc.f90:1-133 + ADJFLAM_DIST
 * adjgrad.f90:88-145 + SAXPY adjgrad.f90:76): derivative in Vp ('PP') or Vs
 * ('SS') at the inversion anchors of GENGMASK, density-normalised element
 * operator DKM_VPVS, ELEM_WTS weighting, COMPLEX*8 virtual forces.  wave and
 * adjlam are COMPLEX*8 [NDOF] device arrays, gradl REAL*4 [NNPINV] device
 * array updated in place.  accumulate = 0 keeps the reference's behaviour of
 * keeping only the last connected element's force (vforce25.f:274-280). */
int fem25_ref_gradient_dev(fem25_ctx *ctx, const char *cinvtype, double vpvs, double freq,
                           double py, const float *wave, const float *adjlam, int accumulate,
                           float *gradl, void *stream);
int fem25_ref_gradient_info(fem25_ctx *ctx, int *nnpinv, long long *nz_fdist,
                            int *maskg /* [NNPG], nullable */);
/* Host-buffer form of the same pair for the call sites of CFMAT_DIST +
 * ADJGRAD (funcgradh.f90:279-295): wave and adjlam host COMPLEX*8 [NDOF],
 * gradl host REAL*4 [NNPINV] updated in place (GRADL of ADJGRAD).
 * Synchronous. */
int fem25_cfmat_adjgrad(fem25_ctx *ctx, const char *cinvtype, double vpvs, double freq, double py,
                        const float *wave, const float *adjlam, int accumulate, float *gradl);

/* Post-processing of the reduced gradient in FUNCGRADH25
 * (funcgradh.f90:436-443), on device arrays in place:
 * fem25_wtgrad_dev is WTGRAD (gengmask.f90:384-416),
 * GRAD(IA35) = GRAD(IA35) * WGRAD(IA35) for na35 REAL*4 values;
 * fem25_avgrad_dev / fem25_avgrad8_dev are AVGRAD / AVGRAD8
 * (gengmask.f90:1202-1332): ncasc cascades of replacing every inversion
 * anchor's value by the mean over the inversion anchors of its connected
 * elements (MCONN, IENG, MASKG of GENGMASK, as fem25_ref_gradient_info
 * reports them), for nvinv (1 or 2) values per anchor, grad REAL*4 /
 * REAL*8 [NNPINV * nvinv] with index (inpinv - 1) * nvinv + ivinv.  The
 * first AVGRAD call builds the GENGMASK tables (outside any capture). */
int fem25_wtgrad_dev(fem25_ctx *ctx, int na35, const float *wgrad, float *grad, void *stream);
int fem25_avgrad_dev(fem25_ctx *ctx, int nvinv, int ncasc, float *grad, void *stream);
int fem25_avgrad8_dev(fem25_ctx *ctx, int nvinv, int ncasc, double *grad, void *stream);

/* Virtual forces of VFORCE25_2 (vforce25.f:373-607) with the alpha / beta
 * derivative matrices of DABMKISOB25 (dstiff25.f:1-203), the convention of
 * the reference's Gauss-Newton / Hessian routines (qpmfree.f90:1119): for
 * every inversion anchor p, F_p(row) = sum over the connected elements (MCONN
 * order, no element weights, no reset between elements) of
 * CMPLX(DCMPLX(DMD,0) + DKD)(row,col) * WAVE(col) in COMPLEX*8.  cinvtype
 * 'PP', 'SS' or 'PS'; fmat COMPLEX*8 [nvinv][NZ_FDIST] on the device with the
 * CSC pattern of fem25_ref_gradient_info (alpha first for 'PS'). */
int fem25_ref_vforce2_dev(fem25_ctx *ctx, const char *cinvtype, double freq, double py,
                          const float *wave, float *fmat, void *stream);

/* Drop-in for MET225_MOD (qpmfree.f90:1000-1250), the Hessian-vector terms
 * of the reference's truncated-Newton inner loop (QPMFREE): for every
 * inversion anchor, with the DABMKISOB25 alpha / beta derivative matrices of
 * its connected elements weighted by ELEM_WTS,
 *   P1BUF(ia) = -sum_rows REAL(CONJG(T1) * NU),  T1 = sum_e w_e dS_e WAVE
 *   P2BUF(ia) = -sum_rows REAL(CONJG(T2) * ADJLAM), T2 = sum_e w_e dS_e ALPHA
 * in COMPLEX*8 / REAL*4, ia = (inpinv - 1) * nvinv + ivinv (alpha first for
 * 'PS').  As in the reference the T columns are nulled inside the element
 * loop, so only the last connected element contributes (accumulate = 0);
 * accumulate = 1 sums every element.  adjlam, nu, alpha, wave: COMPLEX*8
 * [NDOF]; p1buf, p2buf: REAL*4 [nnpinv * nvinv] (overwritten); device. */
int fem25_ref_met225_dev(fem25_ctx *ctx, const char *cinvtype, double freq, double py,
                         const float *adjlam, const float *nu, const float *alpha,
                         const float *wave, int accumulate, float *p1buf, float *p2buf,
                         void *stream);

/* Drop-in for the kernels of CADJ_NU_ALPHA (qpmfree.f90:622-996), the
 * second-order adjoint step of the truncated-Newton inner loop, for a model
 * perturbation v (REAL*4 [nnpinv * nvinv], device): with the DABMKISOB25
 * alpha / beta blocks of every (inversion anchor, connected element) pair
 * weighted by CWGHT = SNGL(ELEM_WTS) * V(ia), in COMPLEX*8 and the
 * reference's summation order,
 *   rhsbnu(JDOF) = sum ADJLAM(IDOF) * CONJG(CWGHT * dS(IDOF, JDOF))
 *   rhsalp(IDOF) = sum CWGHT * dS(IDOF, JDOF) * WAVE(JDOF)
 *   p3(ia)       = -sum_rows REAL(CONJG(TEMP) * ADJLAM)
 * (TEMP as rhsalp restricted to the anchor's elements; only the last
 * connected element survives unless accumulate = 1, as in the reference).
 * The two MUMPS solves stay with the caller: NU = CONJG(S^-T CONJG(rhsbnu)),
 * ALPHA = S^-1 rhsalp (fem25_dense_solve_dev on small meshes).  The first
 * call builds the pair lists and a weighted-block workspace of
 * pairs x nvinv x 75^2 COMPLEX*8 (about 4 pairs per anchor).  adjlam, wave,
 * rhsbnu, rhsalp: COMPLEX*8 [NDOF] (outputs overwritten); device. */
int fem25_ref_cadj_nu_alpha_dev(fem25_ctx *ctx, const char *cinvtype, double freq, double py,
                                const float *v, const float *adjlam, const float *wave,
                                int accumulate, float *rhsbnu, float *rhsalp, float *p3,
                                void *stream);

/* Drop-in for the products of PCHADJ (pchadj.f90:1-330) that follow its
 * Green's-function solve (G^T = S^-T (-A^T) for the nrhs = NDIM x NREC
 * receiver components, which the caller's solver provides): per inversion
 * anchor, the Jacobian block JACL(irhs, v) = sum_rows G(irhs, row) F(row, v)
 * in COMPLEX*8, and the block-diagonal preconditioner update
 * HESSB += REAL(JACL^H JACL) (CGEMM order of the reference BLAS, then
 * SAXPY).  grns: COMPLEX*8 [nrhs][NDOF]; fmat: COMPLEX*8 [nvinv][NZ_FDIST]
 * (the forces of fem25_ref_gradient_dev / _vforce2_dev); hessb: REAL*4
 * [nnpinv * nvinv^2] updated in place, block (col, iv, jv) at
 * (col * nvinv + iv) * nvinv + jv; jacl (nullable, the LGNEWT Jacobian):
 * COMPLEX*8 [nnpinv * nvinv][nrhs].  nrhs * nvinv <= 25 600.  Device. */
int fem25_ref_pchadj_dev(fem25_ctx *ctx, int nvinv, int nrhs, const float *grns,
                         const float *fmat, float *hessb, float *jacl, void *stream);

/* ---- forward misfit + adjoint source ---------------------------------------
 * Options of fem25_misfit_dev and fem25_misfit_noalloc_dev, kept by the
 * context (the reference's INV_INFO fields; defaults NORM 2, IRESTP 3,
 * IBPHASE 0, no thresholds, no phase-jump tests):
 *   norm     NORM of COBJ4 / BPRESID4 (objfn.f:5-175, :757-847):
 *            1 L1, 2 L2, 3 Huber, 4 L1/L2 combination;
 *   irestp   IRESTP of CRESID (objfn.f:953-1012): 1 phase only,
 *            2 amplitude only, 3 phase and amplitude;
 *   ibphase  IBPHASE of HDIFFER (adjgrad.f90:528-566): 0 none, 1 sqrt(-iw),
 *            2 -sqrt(-iw), 3 sqrt(iw), 4 -sqrt(iw), 5 iw, 6 i;
 *   eps, thresh  COBJ4's EPS = EPSS * CRESMN and THRESH = THRESHS * CRESMN
 *            (NORM 3 and 4), computed by the caller over its data set;
 *   dtmax    BPRESID4's DTMAX (L2: residuals whose phase difference is a
 *            time shift above dtmax are zeroed; 0 = off);
 *   dtmax_obj COBJ4's DTMAX (L2; FUNCGRADH25 passes 0, funcgradh.f90:405).
 * As in the reference, BPRESID4 uses EPS = 0 for every norm
 * (objfn.f:795-797): its NORM 3 residual equals the L1 one unless W DIF = 0,
 * and its NORM 4 residual is not finite.  IRESTP 1 and the DTMAX tests take
 * phases with the device's atan2f / cosf / sinf. */
int fem25_misfit_options(fem25_ctx *ctx, int norm, int irestp, int ibphase, float eps,
                         float thresh, float dtmax, float dtmax_obj);

/* EXRESP25D (locrec2d.f:867-925) + rotation + CRESID + BPRESID4 + COBJ4 +
 * RESID_DRHS with HDIFFER (adjgrad.f90:448-566) for nsrc solutions at once.
 * sol: COMPLEX*8 [nsrc][NDOF] device; mrdof: MRDOF(3,NREC) host;
 * yrec[NREC], recv COMPLEX*8 (3,NREC), obs COMPLEX*8 [nsrc](3,NREC),
 * wghts REAL*4 [nsrc](3,NREC) host; outputs: est COMPLEX*8 [nsrc](3,NREC)
 * host, rhs COMPLEX*8 [nsrc][NDOF] device (conjugated, ready for the
 * transpose solve), misfit[nsrc] host (the source's sum of COBJ4's terms,
 * for L2 sum |w|^2 |obs-est|^2, not halved). */
int fem25_misfit_dev(fem25_ctx *ctx, int nsrc, int nrec, const int *mrdof, const double *yrec,
                     double freq, double py, double azmod, const float *recv, const float *sol,
                     const float *obs, const float *wghts, float *est, float *rhs, float *misfit,
                     void *stream);

/* The pass after the solve, fused into one kernel for nsrc sources: ADDBLK
 * (bielak_utils.f:1116-1125; sol += ue on the 'E' DOFs, in place), then
 * EXRESP25D and the misfit / adjoint source of fem25_misfit_dev on the
 * updated solutions (the three steps at funcgradh.f90:248-263 and
 * adjgrad.f90:288-323).  Arguments as fem25_misfit_dev plus ue and sol
 * (COMPLEX*8 [nsrc][NDOF] device, sol updated); results bit-identical to
 * fem25_addblk_dev followed by fem25_misfit_dev.  nrec <=
 * FEM25_POSTSOLVE_MAX_REC; the receiver bitmap is rebuilt (synchronously)
 * when MRDOF differs from the previous call's. */
#define FEM25_POSTSOLVE_MAX_REC 16384
int fem25_postsolve_dev(fem25_ctx *ctx, int nsrc, int nrec, const int *mrdof, const double *yrec,
                        double freq, double py, double azmod, const float *recv, const float *ue,
                        float *sol, const float *obs, const float *wghts, float *est, float *rhs,
                        float *misfit, void *stream);

/* The same misfit and adjoint source without any device allocation, for
 * callers that must not allocate device memory while they run: an inversion
 * loop that has given the rest of HBM to a sparse direct solver's factors, or
 * one that cannot take the device-wide synchronisation that cudaMalloc and
 * cudaFree imply between frequencies.  No counterpart in the reference (it
 * has no device memory); it computes what fem25_misfit_dev computes, with
 * bit-identical outputs.
 * Differences from fem25_misfit_dev: obs, wghts, est and misfit are DEVICE
 * arrays here (same layouts); mrdof, yrec and recv stay host arrays and are
 * copied into a fixed device scratch before the call returns.
 * Limits: nrec <= FEM25_NOALLOC_MAX_REC and nsrc * nrec <=
 * FEM25_NOALLOC_MAX_SRC_REC; larger calls return FEM25_ERR_ARG with a message.
 * The scratch (about 3.1 MB) is one static array per device, shared by every
 * context on that device: calls that overlap in time on one device (two
 * threads, or two streams with no ordering between them) race on it and give
 * wrong results.  The first call on each device sets the scratch up (looks up
 * its address, which may load the library's device code); make that first
 * call before any stream capture begins.  That address is kept for the life
 * of the process: do not use this entry point across a cudaDeviceReset.
 * The receiver tables are staged from host buffers that live only during the
 * call, so a call on a stream that is being captured returns FEM25_ERR_ARG. */
#define FEM25_NOALLOC_MAX_REC 2048
#define FEM25_NOALLOC_MAX_SRC_REC 262144
int fem25_misfit_noalloc_dev(fem25_ctx *ctx, int nsrc, int nrec, const int *mrdof,
                             const double *yrec, double freq, double py, double azmod,
                             const float *recv, const float *sol, const float *obs,
                             const float *wghts, float *est, float *rhs, float *misfit,
                             void *stream);

/* ---- profiling ----------------------------------------------------------------
 * With profiling enabled the library records CUDA events on the launching
 * stream around its dominant kernels; fem25_profile_ms returns the duration
 * of the last launch: which = 0 the batched streaming kernel, which = 1 the
 * plain element + gather kernels of fem25_assemble_dev. */
/* The choices of the per-context autotuners, -1 before the first call that
 * tunes them: the streaming-assembly variant (0-2: 1, 2, 4 entries per
 * thread; 3: software-pipelined; 4, 5: all systems of a 64 / 128-entry chunk
 * staged for bulk stores; 6, 7: 256 / 512-entry staging ring, 16 systems per
 * launch; 8, 9: 512 / 256-entry staging ring, up to min(1024, nslots)
 * systems per launch)
 * and the source tile of the FP64 gradient (2, 4 or 8 sources per
 * shared-memory pass). */
int fem25_tuning(const fem25_ctx *ctx, int *stream_variant, int *grad_tile);

/* Waits for the stream and reports what the context's kernels recorded on
 * the device since the last check: FEM25_ERR_JACOBIAN for an element whose
 * Jacobian the gradient kernels found undefined or negative, FEM25_ERR_CUDA
 * for a bounded pipeline wait of a tensor-core gradient kernel that ran out
 * (that launch's results are invalid).  The asynchronous entry points
 * (gradient, batch) do not wait; call this where the stream is synchronised
 * anyway (after a gradient, before reading it back). */
int fem25_sync_status(fem25_ctx *ctx, void *stream);

/* Test hook of the bounded waits above (no counterpart in the reference):
 * limit_cycles > 0 sets the SM clocks a pipeline wait of the tensor-core
 * gradient kernels may take before it gives up (<= 0: the default, about half
 * a second); inject = 1 makes the next launches withhold one producer
 * arrival in their first CTA, so that a wait runs out, the launch drains and
 * fem25_sync_status reports FEM25_ERR_CUDA (the covariances accumulated since
 * the last finalize are then discarded).  inject = 0 restores normal runs. */
int fem25_test_waits(fem25_ctx *ctx, long long limit_cycles, int inject);
int fem25_profile_enable(fem25_ctx *ctx, int enable);
int fem25_profile_ms(fem25_ctx *ctx, int which, double *ms);

#ifdef __cplusplus
}
#endif
#endif /* FEM25GPU_H */
