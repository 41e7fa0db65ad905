// csp_noalloc.cu -- per-domain min / max / sum of one FP32 field with no device
// allocation (csp_reduce_field_noalloc in include/csparks.h).
//
// Some callers cannot allocate device memory: a plugin hosted in a process whose
// framework has reserved the device memory for its own pool, or code that runs where a
// cudaMalloc would stall (it synchronises the device) such as a latency-bound loop.  This
// entry point takes the caller's device buffers for the field, its domain ids and the
// result, and keeps its block partials in a fixed file-scope device array instead of an
// allocation.  It computes the same reductions as csp_reduce_outputs.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdio>
#include <mutex>

#include "../../include/csparks.h"
#include "csp_device.cuh"   // csp::DOMAIN_BITS: the domain-id bits of a domain byte

namespace {

constexpr int NOALLOC_BLOCKS = 592;                 // 148 SMs x 4 resident blocks
constexpr int NOALLOC_THREADS = 256;
constexpr int ND = CSP_MAX_DOMAINS;

// Block partials: [block][min, max, sum][domain].  Every call writes all the slots it then
// reads, so nothing has to start at zero; the contents of the previous call stay until then.
static __device__ __align__(256) double g_partials[NOALLOC_BLOCKS * 3 * ND];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_partials_ptr[MAX_DEVICES] = {nullptr};

__global__ void __launch_bounds__(NOALLOC_THREADS) k_noalloc_partial(const float* __restrict__ u,
                                                                     const unsigned char* __restrict__ dom,
                                                                     long long n, int nd,
                                                                     double* __restrict__ part) {
  double mn[ND], mx[ND], sm[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) { mn[d] = FLT_MAX; mx[d] = FLT_MIN; sm[d] = 0.0; }
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int d = dom[i] & csp::DOMAIN_BITS;
    const double v = (double)u[i];
#pragma unroll
    for (int dd = 0; dd < ND; dd++)
      if (dd == d) {
        mn[dd] = v < mn[dd] ? v : mn[dd];
        mx[dd] = v > mx[dd] ? v : mx[dd];
        sm[dd] += v;
      }
  }
  __shared__ double red[3][ND][NOALLOC_THREADS];
#pragma unroll
  for (int d = 0; d < ND; d++) { red[0][d][threadIdx.x] = mn[d]; red[1][d][threadIdx.x] = mx[d]; red[2][d][threadIdx.x] = sm[d]; }
  __syncthreads();
  for (int w = NOALLOC_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        double a = red[0][d][threadIdx.x + w];
        if (a < red[0][d][threadIdx.x]) red[0][d][threadIdx.x] = a;
        a = red[1][d][threadIdx.x + w];
        if (a > red[1][d][threadIdx.x]) red[1][d][threadIdx.x] = a;
        red[2][d][threadIdx.x] += red[2][d][threadIdx.x + w];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < nd) {
    const int d = threadIdx.x;
    part[(blockIdx.x * 3 + 0) * ND + d] = red[0][d][0];
    part[(blockIdx.x * 3 + 1) * ND + d] = red[1][d][0];
    part[(blockIdx.x * 3 + 2) * ND + d] = red[2][d][0];
  }
}

__global__ void k_noalloc_final(const double* __restrict__ part, int nblk, int nd, double dV,
                                double* __restrict__ out) {
  const int d = threadIdx.x;
  if (d >= nd) return;
  double mn = FLT_MAX, mx = FLT_MIN, sm = 0.0;
  for (int b = 0; b < nblk; b++) {
    const double a = part[(b * 3 + 0) * ND + d], c = part[(b * 3 + 1) * ND + d];
    mn = a < mn ? a : mn;
    mx = c > mx ? c : mx;
    sm += part[(b * 3 + 2) * ND + d];
  }
  out[0 * nd + d] = mn;
  out[1 * nd + d] = mx;
  out[2 * nd + d] = sm * dV;
}

}  // namespace

// Address of the partials array on the current device, looked up once per device and kept
// for the life of the process.  A cudaDeviceReset reloads the module and may move the
// array, so this entry point is not supported on a device after cudaDeviceReset.
static int noalloc_setup(double** ptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return CSP_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_partials_ptr[dev]) {
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_partials);
    if (e != cudaSuccess || !p) {
      fprintf(stderr, "csp_reduce_field_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
      return CSP_ECUDA;
    }
    g_partials_ptr[dev] = p;
  }
  *ptr = g_partials_ptr[dev];
  return CSP_OK;
}

extern "C" int csp_reduce_field_noalloc(const float* field, const uint8_t* domains, int64_t n,
                                        int32_t num_domains, double dV, double* out, void* stream) {
  if (!field || !domains || !out || n < 1) return CSP_EINVAL;
  if (num_domains < 1 || num_domains > CSP_NOALLOC_MAX_DOMAINS) {
    fprintf(stderr, "csp_reduce_field_noalloc: num_domains %d outside 1..%d (size of the fixed scratch)\n",
            num_domains, CSP_NOALLOC_MAX_DOMAINS);
    return CSP_ERANGE;
  }
  if (n > CSP_NOALLOC_MAX_VOXELS) {
    fprintf(stderr, "csp_reduce_field_noalloc: %lld voxels above the maximum %lld\n", (long long)n,
            (long long)CSP_NOALLOC_MAX_VOXELS);
    return CSP_ERANGE;
  }
  double* part = nullptr;
  const int rc = noalloc_setup(&part);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  long long want = (n + NOALLOC_THREADS - 1) / NOALLOC_THREADS;
  const int nblk = (int)(want < NOALLOC_BLOCKS ? want : NOALLOC_BLOCKS);
  k_noalloc_partial<<<nblk, NOALLOC_THREADS, 0, s>>>(field, domains, n, num_domains, part);
  k_noalloc_final<<<1, 32, 0, s>>>(part, nblk, num_domains, dV, out);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CSP_OK : CSP_ECUDA;
}
