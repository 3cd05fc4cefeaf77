// noalloc.cu -- convergence norm for callers that cannot allocate device
// memory.
//
// desalm_mg_residual() reduces |q - qold| through a partial-sum buffer that
// the context allocates with cudaMalloc when it is created.  Some callers
// cannot do that: code running while a CUDA stream is being captured into a
// graph (cudaMalloc is not a capturable operation), Fortran drivers whose
// device memory is owned by a pool or another runtime, and host paths that
// must not touch the CUDA allocator at all (for example under strict memory
// accounting).  desalm_mg_residual_noalloc() computes the same five values
// from caller-owned device arrays and keeps its scratch in a fixed, file-scope
// device array instead.
//
// The scratch array lives in the library image: every GPU that loads the
// library holds it (DESALM_NOALLOC_MAX_PARTIALS * 5 + 5 doubles, about
// 2.5 MiB) until the process exits.  All calls share it, so calls that
// overlap on the GPU (two streams, or two host threads) race on it and must
// be serialised by the caller.  Each call overwrites every slot it reads, so
// nothing is carried over from the previous call's contents.
#include <cuda_runtime.h>
#include <cmath>
#include "desalm.h"

#define DESALM_NOALLOC_MAX_PARTIALS 65536   // one partial per block of 2048 interior nodes
#define DESALM_NOALLOC_NODES_PER_BLOCK 2048

namespace {

static __device__ __align__(256) double g_noalloc_scratch[DESALM_NOALLOC_MAX_PARTIALS * 5 + 5];

// Device address of g_noalloc_scratch, looked up once per device (the
// host-side symbol is only a stand-in, not a device address).
static double* g_scratch_ptr[64] = {nullptr};

__global__ void k_noalloc_partial(const double* q, const double* qold, int im, int jm, int km, long n_int, double* part) {
  __shared__ double sh[5][256];
  double acc[5] = {0, 0, 0, 0, 0};
  const int ni = im - 2, nj = jm - 2;
  const long N = (long)im * jm * km;
  const long first = (long)blockIdx.x * DESALM_NOALLOC_NODES_PER_BLOCK;
  for (int r = 0; r < DESALM_NOALLOC_NODES_PER_BLOCK / 256; ++r) {
    long t = first + r * 256 + threadIdx.x;
    if (t >= n_int) break;
    const int i = int(t % ni) + 1;
    const long rr = t / ni;
    const int j = int(rr % nj) + 1;
    const int k = int(rr / nj) + 1;
    const long l = i + (long)im * (j + (long)jm * k);
    for (int m = 0; m < 5; ++m) acc[m] += fabs(q[m * N + l] - qold[m * N + l]);
  }
  for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] += sh[m][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) part[blockIdx.x * 5 + m] = sh[m][0];
}

__global__ void k_noalloc_final(const double* part, int nblk, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int m = 0; m < 5; ++m) {
    double s = 0;
    for (int b = 0; b < nblk; ++b) s += part[b * 5 + m];
    out[m] = s;
  }
}

}  // namespace

extern "C" int desalm_mg_residual_noalloc(const double* q, const double* qold, int im, int jm, int km,
                                          double res[5], void* stream) {
  if (im < 3 || jm < 3 || km < 3) return DESALM_EINVAL;
  const long n_int = (long)(im - 2) * (jm - 2) * (km - 2);
  const long nblk = (n_int + DESALM_NOALLOC_NODES_PER_BLOCK - 1) / DESALM_NOALLOC_NODES_PER_BLOCK;
  // more than 134,217,728 interior nodes do not fit the fixed scratch
  if (nblk > DESALM_NOALLOC_MAX_PARTIALS) return DESALM_ENOMEM;
  // every pointer is checked before anything is launched
  if (!q || !qold || !res) return DESALM_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DESALM_ECUDA;
  if (!g_scratch_ptr[dev]) {
    // first call on this device: resolve the scratch's device address (must
    // happen before any stream capture that includes this entry point)
    double* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) return DESALM_ECUDA;
    g_scratch_ptr[dev] = p;
  }
  double* part = g_scratch_ptr[dev];
  double* sums = part + DESALM_NOALLOC_MAX_PARTIALS * 5;
  cudaStream_t s = (cudaStream_t)stream;
  k_noalloc_partial<<<(unsigned)nblk, 256, 0, s>>>(q, qold, im, jm, km, n_int, part);
  k_noalloc_final<<<1, 32, 0, s>>>(part, (int)nblk, sums);
  if (cudaGetLastError() != cudaSuccess) return DESALM_ECUDA;
  double h[5];
  if (cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DESALM_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return DESALM_ECUDA;
  const double tnu = double(n_int);
  for (int m = 0; m < 5; ++m) res[m] = std::log10(h[m] / tnu);
  return 0;
}
