// fem25_misfit_noalloc_dev: the forward misfit and adjoint source of
// fem25_misfit_dev for callers that must not allocate device memory while
// they run.  Two kinds of caller need it: an inversion loop that has handed
// the rest of HBM to a sparse direct solver's factors (an allocation of a
// few MB between frequencies can then fail), and a loop that cannot take the
// device-wide synchronisation that cudaMalloc / cudaFree imply between
// frequencies.  The per-call device buffers of fem25_misfit_dev (receiver
// tables, the COBJ4 partial sums, copies of obs / wghts / est / misfit)
// become, here, one fixed scratch array in the library's device image plus
// caller-owned device arrays.
//
// Scratch: g_misfit_scratch, a file-scope static __device__ array of
// kScratchBytes (about 3.1 MB), laid out as
//   mrdof  int   [3 * kMaxRec]      receiver DOF numbers (MRDOF(3,NREC))
//   trig   float4[kMaxRec]          cos/sin of +-omega*py*yrec per receiver
//   recv   float2[3 * kMaxRec]      receiver response factors
//   part   float [3 * kMaxSrcRec]   per (source, receiver, component) misfit terms
// Nothing in it has to start at zero: every entry a call reads was written
// earlier in the same call (the tables by the host copies, each partial by
// k_misfit before k_misfit_sum sums it).
//
// Set-up: the first call on each device (with that device current) looks up
// the scratch's device address with cudaGetSymbolAddress and caches it; this
// may load the library's device code on that device, so make the first call
// before any stream capture begins.  The cached address belongs to the
// device's primary context: after a cudaDeviceReset in the process (or a
// library that destroys the primary context) it is stale, so the entry point
// must not be used across a device reset.
//
// Host staging: the receiver tables pass through stack buffers of this call
// with cudaMemcpyAsync, so a call on a stream that is being captured returns
// FEM25_ERR_ARG (a recorded copy would read those buffers after the call has
// returned).
//
// Concurrency: the scratch is one array per device, shared by every context
// on it.  Calls that overlap in time on one device (two host threads, or two
// streams without an ordering between them) race on it and return wrong
// results; serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

#include "ctx.cuh"

using namespace fem25;

struct fem25_ctx {
  Ctx c;
};

namespace {

constexpr int kMaxRec = FEM25_NOALLOC_MAX_REC;
constexpr long long kMaxSrcRec = FEM25_NOALLOC_MAX_SRC_REC;
constexpr size_t kOffMrdof = 0;
constexpr size_t kOffTrig = kOffMrdof + sizeof(int) * 3 * kMaxRec;
constexpr size_t kOffRecv = kOffTrig + sizeof(float4) * kMaxRec;
constexpr size_t kOffPart = kOffRecv + sizeof(float2) * 3 * kMaxRec;
constexpr size_t kScratchBytes = kOffPart + sizeof(float) * 3 * kMaxSrcRec;
static_assert(kOffTrig % 16 == 0 && kOffRecv % 16 == 0 && kOffPart % 16 == 0, "scratch alignment");

static __device__ __align__(256) unsigned char g_misfit_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device `dev`, looked up once.
cudaError_t scratch_on(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_misfit_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

int fail(Ctx *c, int code, const char *msg) {
  if (c) c->err = msg;
  std::fprintf(stderr, "fem25gpu: %s\n", msg);
  return code;
}

int cuda_fail(Ctx *c, cudaError_t e, const char *where) {
  char buf[256];
  std::snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
  return fail(c, FEM25_ERR_CUDA, buf);
}

// receivers staged per host->device copy (13 KB of stack)
constexpr int kChunk = 256;

}  // namespace

extern "C" int fem25_misfit_noalloc_dev(fem25_ctx *h, int nsrc, int nrec, const int *mrdof,
                                        const double *yrec, double freq, double py, double azmod,
                                        const float *recv, const float *sol, const float *obs,
                                        const float *wghts, float *est, float *rhs, float *misfit,
                                        void *stream) {
  if (!h || nsrc <= 0 || nrec <= 0 || !mrdof || !yrec || !recv || !sol || !obs || !wghts || !est ||
      !rhs || !misfit)
    return FEM25_ERR_ARG;
  Ctx *c = &h->c;
  if (nrec > kMaxRec) {
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "misfit_noalloc: nrec = %d exceeds the fixed scratch limit "
                  "FEM25_NOALLOC_MAX_REC = %d",
                  nrec, kMaxRec);
    return fail(c, FEM25_ERR_ARG, buf);
  }
  if ((long long)nsrc * nrec > kMaxSrcRec) {
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "misfit_noalloc: nsrc * nrec = %lld exceeds the fixed scratch limit "
                  "FEM25_NOALLOC_MAX_SRC_REC = %lld",
                  (long long)nsrc * nrec, kMaxSrcRec);
    return fail(c, FEM25_ERR_ARG, buf);
  }
  // the checks of fem25_misfit_dev: DOFs in range and no DOF shared by two
  // receiver components (they would race in the right-hand side)
  {
    int seen[3 * kMaxRec];
    int n = 0;
    for (int k = 0; k < 3 * nrec; k++) {
      if (mrdof[k] < 0 || mrdof[k] > c->ndof)
        return fail(c, FEM25_ERR_ARG, "misfit: MRDOF entry out of range");
      if (mrdof[k] > 0) seen[n++] = mrdof[k];
    }
    std::sort(seen, seen + n);
    if (std::adjacent_find(seen, seen + n) != seen + n)
      return fail(c, FEM25_ERR_ARG, "misfit: two receiver components share a DOF");
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(c, e, "set device");
  cudaStream_t st = (cudaStream_t)stream;
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess)
      return cuda_fail(c, e, "misfit_noalloc: stream status");
    if (cs != cudaStreamCaptureStatusNone)
      return fail(c, FEM25_ERR_ARG,
                  "misfit_noalloc: the stream is being captured; the receiver tables are "
                  "staged from host buffers that do not outlive the call");
  }
  unsigned char *base = nullptr;
  if ((e = scratch_on(c->device, &base)) != cudaSuccess) return cuda_fail(c, e, "misfit scratch");
  int *d_mrdof = reinterpret_cast<int *>(base + kOffMrdof);
  float *d_trig = reinterpret_cast<float *>(base + kOffTrig);
  float *d_recv = reinterpret_cast<float *>(base + kOffRecv);
  float *d_part = reinterpret_cast<float *>(base + kOffPart);
  // receiver tables: staged through pageable stack buffers, so the caller's
  // host arrays are no longer needed when the call returns
  const double omega = 6.2831853071795862 * freq;
  int hm[3 * kChunk];
  float ht[4 * kChunk], hr[6 * kChunk];
  for (int r0 = 0; r0 < nrec; r0 += kChunk) {
    const int nr = std::min(kChunk, nrec - r0);
    for (int ir = 0; ir < nr; ir++) {
      const double y = yrec[r0 + ir];
      float ph = (float)(omega * py * y);
      float ph2 = -(float)(omega * py * y);
      ht[4 * ir + 0] = cosf(ph);
      ht[4 * ir + 1] = sinf(ph);
      ht[4 * ir + 2] = cosf(ph2);
      ht[4 * ir + 3] = sinf(ph2);
    }
    std::copy(mrdof + 3 * (size_t)r0, mrdof + 3 * (size_t)(r0 + nr), hm);
    std::copy(recv + 6 * (size_t)r0, recv + 6 * (size_t)(r0 + nr), hr);
    if ((e = cudaMemcpyAsync(d_mrdof + 3 * (size_t)r0, hm, sizeof(int) * 3 * nr,
                             cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_trig + 4 * (size_t)r0, ht, sizeof(float) * 4 * nr,
                             cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_recv + 6 * (size_t)r0, hr, sizeof(float) * 6 * nr,
                             cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return cuda_fail(c, e, "misfit receiver tables");
  }
  e = launch_misfit_part(c, nsrc, nrec, d_mrdof, d_trig, freq, azmod, d_recv, sol, obs, wghts, est,
                         rhs, d_part, misfit, st);
  if (e != cudaSuccess) return cuda_fail(c, e, "misfit");
  return FEM25_OK;
}
