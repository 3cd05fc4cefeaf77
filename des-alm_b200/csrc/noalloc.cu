// noalloc.cu -- convergence norm for callers that cannot allocate device
// memory.
//
// desalm_mg_residual() reduces |q - qold| through a partial-sum buffer that
// the context allocates with cudaMalloc when it is created.  Some callers
// cannot do that: Fortran drivers whose device memory is owned by another
// runtime or pool allocator (a CUDA Fortran or OpenACC runtime that hands out
// device arrays and must see every allocation), and processes that run under
// a fixed device-memory budget where any allocation outside the host's own
// allocator is an error.  desalm_mg_residual_noalloc() computes the same five
// values from caller-owned device arrays and keeps its scratch in a fixed,
// file-scope device array instead; it calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// The scratch array lives in the library image: every GPU that loads the
// library holds it (DESALM_NOALLOC_MAX_PARTIALS * 5 + 5 doubles, about
// 2.5 MiB) until the process exits.  All calls share it, so calls that
// overlap on the GPU (two streams, or two host threads) race on it and must
// be serialised by the caller.  Each call overwrites every slot it reads
// before reading it, so nothing is carried over from the previous call.
//
// In host code the array's name is only a host-side stand-in, not a device
// address.  The first call on each device, with that device current, looks
// up the array's device address with cudaGetSymbolAddress and keeps it for
// the process; later calls on that device reuse it.  That first call should
// come before any stream capture, and cudaDeviceReset after it is not
// supported (the reset unloads the module and the kept address dies with
// it).  The lookup is guarded by a mutex, so host threads may make their
// first calls at once.
#include <cuda_runtime.h>
#include <cmath>
#include <mutex>
#include "desalm.h"

#define DESALM_NOALLOC_MAX_PARTIALS 65536   // one partial per block of 2048 interior nodes
#define DESALM_NOALLOC_NODES_PER_BLOCK 2048
#define DESALM_NOALLOC_MAX_DEVICES 64

namespace {

static __device__ __align__(256) double g_noalloc_scratch[DESALM_NOALLOC_MAX_PARTIALS * 5 + 5];

// Device address of g_noalloc_scratch per device, looked up once.
static double* g_scratch_ptr[DESALM_NOALLOC_MAX_DEVICES] = {nullptr};
static std::mutex g_scratch_mu;

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

// One block of 256 threads: thread t sums partials t, t + 256, ... in
// order, then a fixed tree adds the 256 sums, so the result does not depend
// on timing and repeats bit for bit.
__global__ void __launch_bounds__(256) k_noalloc_final(const double* part, int nblk, double* out) {
  __shared__ double sh[5][256];
  double acc[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblk; b += 256)
    for (int m = 0; m < 5; ++m) acc[m] += part[b * 5 + m];
  for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] += sh[m][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 5) out[threadIdx.x] = sh[threadIdx.x][0];
}

// The scratch's device address on the current device (resolved on the first
// call there); nullptr on a CUDA error.
double* scratch_on_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= DESALM_NOALLOC_MAX_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) return nullptr;
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
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
  double* part = scratch_on_current_device();
  if (!part) return DESALM_ECUDA;
  double* sums = part + DESALM_NOALLOC_MAX_PARTIALS * 5;
  cudaStream_t s = (cudaStream_t)stream;
  k_noalloc_partial<<<(unsigned)nblk, 256, 0, s>>>(q, qold, im, jm, km, n_int, part);
  k_noalloc_final<<<1, 256, 0, s>>>(part, (int)nblk, sums);
  if (cudaGetLastError() != cudaSuccess) return DESALM_ECUDA;
  double h[5];
  if (cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DESALM_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return DESALM_ECUDA;
  const double tnu = double(n_int);
  for (int m = 0; m < 5; ++m) res[m] = std::log10(h[m] / tnu);
  return 0;
}
