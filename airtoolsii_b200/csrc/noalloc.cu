// airt_residual_noalloc: the SIRT forward residual (r = b - A*x, ||r||) for
// callers that cannot allocate device memory.
//
// Who cannot allocate: code that runs inside a host application which owns
// the whole device memory budget through its own pool (a MATLAB MEX session
// sharing the GPU with gpuArray's caching allocator, a serving process that
// pre-reserves HBM), and code that must not call cudaMalloc/cudaFree because
// those calls synchronise the device and stall every other stream of the
// process.  Such a caller already holds the matrix, x, b and r on the device
// and only needs the kernel; this entry point brings its own scratch instead
// of allocating it.
//
// Scratch: one file-scope __device__ array, kNoAllocMaxN FP32 entries for the
// FP32 copy of x that the gather reads, plus one FP64 reduction slot.  Every
// GPU that loads the library holds it (4 MiB + 256 B) until the process
// exits.  A host-side use of the array's name is only a host stand-in, so the
// device address is looked up with cudaGetSymbolAddress once per device (on
// the first call made on that device, with that device current) and passed
// to the kernels.  That first call should therefore come before any CUDA
// stream capture.  All calls share the array and it keeps the last call's
// contents: the reduction slot is cleared at the start of every call, and two
// calls whose work overlaps on the GPU (different streams, no ordering) race
// on it.  Sizes beyond the maximum are rejected with AIRT_ERR_ARG.
#include <mutex>

#include "common.cuh"
#include "spmv.cuh"

namespace airt {
namespace {

constexpr int64_t kNoAllocMaxN = int64_t(1) << 20;  // image pixels (1024 x 1024)
constexpr size_t kNoAllocBytes = (size_t)kNoAllocMaxN * sizeof(float) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[kMaxDevices] = {nullptr};

// x (FP64) -> FP32 gather copy; one thread also clears the reduction slot.
__global__ void k_noalloc_prepare(int64_t n, const double *__restrict__ x, float *__restrict__ x32,
                                  double *__restrict__ acc) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *acc = 0.0;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    x32[j] = (float)x[j];
}

// The forward residual of the SIRT iteration (k_sirt_fwd) without the
// M-weighting: r = b - A*x over the caller's FP32 CSR, ||r||^2 into *acc.
template <int LANES>
__global__ void __launch_bounds__(256) k_noalloc_resid(int64_t m, const int64_t *__restrict__ rp,
                                                       const int *__restrict__ ci,
                                                       const float *__restrict__ rv,
                                                       const float *__restrict__ x32,
                                                       const double *__restrict__ b,
                                                       double *__restrict__ r,
                                                       double *__restrict__ acc) {
  double a = 0.0;
  for_each_segment<LANES>(m, rp, ci, rv, x32, [&](int64_t i, double s, bool lead) {
    if (lead) {
      const double ri = b[i] - s;
      r[i] = ri;
      a += ri * ri;
    }
  });
  a = block_sum<256>(a);
  if (threadIdx.x == 0) atomicAdd(acc, a);
}

__global__ void k_noalloc_finish(const double *__restrict__ acc, double *__restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *out = sqrt(*acc);
}

unsigned char *scratch_address() {
  int dev = 0;
  AIRT_CHECK_CUDA(cudaGetDevice(&dev));
  AIRT_REQUIRE(dev >= 0 && dev < kMaxDevices, "device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    AIRT_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<unsigned char *>(p);
  }
  return g_noalloc_addr[dev];
}

}  // namespace
}  // namespace airt

using namespace airt;

extern "C" int airt_residual_noalloc(int64_t m, int64_t n, const int64_t *d_rp, const int *d_ci,
                                     const float *d_rv, const double *d_x, const double *d_b,
                                     double *d_r, double *d_resnorm, void *cuda_stream) {
  try {
    AIRT_REQUIRE(m >= 0 && n >= 0, "matrix size out of range");
    AIRT_REQUIRE(n <= kNoAllocMaxN,
                 "n = %lld exceeds the no-alloc maximum of %lld unknowns (the static scratch "
                 "holds one FP32 copy of x)",
                 (long long)n, (long long)kNoAllocMaxN);
    AIRT_REQUIRE(d_rp && d_b && d_r && d_resnorm && (n == 0 || d_x) && (m == 0 || (d_ci && d_rv)),
                 "null pointer argument");
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    unsigned char *base = scratch_address();
    float *x32 = reinterpret_cast<float *>(base);
    double *acc = reinterpret_cast<double *>(base + (size_t)kNoAllocMaxN * sizeof(float));
    k_noalloc_prepare<<<grid_for(n > 0 ? n : 1, 256), 256, 0, s>>>(n, d_x, x32, acc);
    AIRT_LAUNCH_CHECK();
    if (m > 0) {
      k_noalloc_resid<8><<<grid_for(m * 8, 256), 256, 0, s>>>(m, d_rp, d_ci, d_rv, x32, d_b, d_r,
                                                              acc);
      AIRT_LAUNCH_CHECK();
    }
    k_noalloc_finish<<<1, 32, 0, s>>>(acc, d_resnorm);
    AIRT_LAUNCH_CHECK();
  } catch (const Status &st) {
    return st.code;
  } catch (...) {
    set_error("unexpected internal error");
    return AIRT_ERR_CUDA;
  }
  return AIRT_OK;
}
