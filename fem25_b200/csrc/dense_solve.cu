// Direct solve of one assembled system on the GPU, for small meshes: the
// complex128 CSR is expanded into a dense column-major matrix and factored by
// LU with partial pivoting (cuSOLVER getrf), then solved for many right-hand
// sides with A, A^T or A^H (getrs).  It stands in for the host MUMPS
// factor/solve hop of the reference (forward solve bielak25.f90:443-446,
// 545-551; transpose adjoint solve adjgrad.f90:327-341) when NDOF is a few
// tens of thousands, so the assemble -> solve -> misfit -> adjoint ->
// gradient loop stays on the device.
#include <cusolverDn.h>

#include "ctx.cuh"

namespace fem25 {

// one warp per CSR row: dense[(col-1)*n + row] = value (1-based JCPTR)
__global__ void k_csr_to_dense(int n, const int *__restrict__ irptr, const int *__restrict__ jcptr,
                               const double2 *__restrict__ csr, double2 *__restrict__ dense) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * blockDim.x / 32;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; r < n; r += nw) {
    for (int j = irptr[r] - 1 + lane; j < irptr[r + 1] - 1; j += 32)
      dense[(size_t)(jcptr[j] - 1) * n + r] = csr[j];
  }
}

struct DenseLU {
  cusolverDnHandle_t h = nullptr;
  cusolverDnParams_t p = nullptr;
  double2 *a = nullptr;        // [n][n] column-major, overwritten by L\U
  int64_t *ipiv = nullptr;     // [n]
  int *info = nullptr;         // device status word
  void *dwork = nullptr;
  size_t dwork_bytes = 0;
  std::vector<char> hwork;
  bool factored = false;
};

static const char *solver_msg(cusolverStatus_t s) {
  switch (s) {
    case CUSOLVER_STATUS_NOT_INITIALIZED: return "cuSOLVER not initialised";
    case CUSOLVER_STATUS_ALLOC_FAILED: return "cuSOLVER allocation failed";
    case CUSOLVER_STATUS_INVALID_VALUE: return "cuSOLVER invalid value";
    case CUSOLVER_STATUS_EXECUTION_FAILED: return "cuSOLVER execution failed";
    default: return "cuSOLVER error";
  }
}

void free_dense(Ctx *c) {
  DenseLU *d = c->dense;
  if (!d) return;
  if (d->a) cudaFree(d->a);
  if (d->ipiv) cudaFree(d->ipiv);
  if (d->info) cudaFree(d->info);
  if (d->dwork) cudaFree(d->dwork);
  if (d->p) cusolverDnDestroyParams(d->p);
  if (d->h) cusolverDnDestroy(d->h);
  delete d;
  c->dense = nullptr;
}

// 0, or the FEM25 status to return with its message in *msg
int dense_factor(Ctx *c, const double *csr128, cudaStream_t st, std::string *msg) {
  const int64_t n = c->ndof;
  if (!c->dense) c->dense = new DenseLU();
  DenseLU *d = c->dense;
  d->factored = false;
  cusolverStatus_t s;
  if (!d->h) {
    if ((s = cusolverDnCreate(&d->h)) || (s = cusolverDnCreateParams(&d->p))) {
      *msg = std::string("dense solve: ") + solver_msg(s);
      return FEM25_ERR_CUDA;
    }
  }
  if ((s = cusolverDnSetStream(d->h, st))) {
    *msg = std::string("dense solve: ") + solver_msg(s);
    return FEM25_ERR_CUDA;
  }
  cudaError_t e;
  if (!d->a) {
    if ((e = cudaMalloc(&d->a, sizeof(double2) * (size_t)n * n)) ||
        (e = cudaMalloc(&d->ipiv, sizeof(int64_t) * n)) || (e = cudaMalloc(&d->info, sizeof(int)))) {
      *msg = std::string("dense solve: ") + cudaGetErrorString(e) +
             " (dense matrix of NDOF^2 complex128)";
      return FEM25_ERR_ALLOC;
    }
  }
  size_t dbytes = 0, hbytes = 0;
  if ((s = cusolverDnXgetrf_bufferSize(d->h, d->p, n, n, CUDA_C_64F, d->a, n, CUDA_C_64F, &dbytes,
                                       &hbytes))) {
    *msg = std::string("dense solve: ") + solver_msg(s);
    return FEM25_ERR_CUDA;
  }
  if (dbytes > d->dwork_bytes) {
    if (d->dwork) cudaFree(d->dwork);
    d->dwork = nullptr;
    d->dwork_bytes = 0;
    if ((e = cudaMalloc(&d->dwork, dbytes))) {
      *msg = std::string("dense solve: workspace: ") + cudaGetErrorString(e);
      return FEM25_ERR_ALLOC;
    }
    d->dwork_bytes = dbytes;
  }
  if (hbytes > d->hwork.size()) d->hwork.resize(hbytes);
  if ((e = cudaMemsetAsync(d->a, 0, sizeof(double2) * (size_t)n * n, st))) {
    *msg = std::string("dense solve: ") + cudaGetErrorString(e);
    return FEM25_ERR_CUDA;
  }
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  k_csr_to_dense<<<nsm * 8, 256, 0, st>>>((int)n, c->d_irptr, c->d_jcptr,
                                          reinterpret_cast<const double2 *>(csr128), d->a);
  if ((e = cudaGetLastError())) {
    *msg = std::string("dense solve: ") + cudaGetErrorString(e);
    return FEM25_ERR_CUDA;
  }
  if ((s = cusolverDnXgetrf(d->h, d->p, n, n, CUDA_C_64F, d->a, n, d->ipiv, CUDA_C_64F, d->dwork,
                            dbytes, hbytes ? d->hwork.data() : nullptr, hbytes, d->info))) {
    *msg = std::string("dense solve: getrf: ") + solver_msg(s);
    return FEM25_ERR_CUDA;
  }
  int info = 0;
  if ((e = cudaMemcpyAsync(&info, d->info, sizeof(int), cudaMemcpyDeviceToHost, st)) ||
      (e = cudaStreamSynchronize(st))) {
    *msg = std::string("dense solve: ") + cudaGetErrorString(e);
    return FEM25_ERR_CUDA;
  }
  if (info != 0) {
    *msg = "dense solve: getrf info = " + std::to_string(info) +
           (info > 0 ? " (exactly singular pivot)" : " (bad argument)");
    return FEM25_ERR_ARG;
  }
  d->factored = true;
  return 0;
}

int dense_solve(Ctx *c, int nrhs, int trans, double *rhs, cudaStream_t st, std::string *msg) {
  DenseLU *d = c->dense;
  if (!d || !d->factored) {
    *msg = "dense solve: no factorisation (call fem25_dense_factor_dev first)";
    return FEM25_ERR_ARG;
  }
  const cublasOperation_t op = trans == 0 ? CUBLAS_OP_N : trans == 1 ? CUBLAS_OP_T : CUBLAS_OP_C;
  cusolverStatus_t s;
  if ((s = cusolverDnSetStream(d->h, st))) {
    *msg = std::string("dense solve: ") + solver_msg(s);
    return FEM25_ERR_CUDA;
  }
  const int64_t n = c->ndof;
  if ((s = cusolverDnXgetrs(d->h, d->p, op, n, nrhs, CUDA_C_64F, d->a, n, d->ipiv, CUDA_C_64F, rhs,
                            n, d->info))) {
    *msg = std::string("dense solve: getrs: ") + solver_msg(s);
    return FEM25_ERR_CUDA;
  }
  return 0;
}

}  // namespace fem25
