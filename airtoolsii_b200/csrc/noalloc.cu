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
// FP32 copy of x that the gather reads, plus one FP64 reduction slot and one
// bad-index flag.  Every GPU that loads the library holds it (4 MiB + 256 B)
// until the process exits.  A host-side use of the array's name is only a
// host stand-in, so the device address is looked up with
// cudaGetSymbolAddress, with the caller's device and context current, and
// passed to the kernels.  The address belongs to a CUDA context, so it is
// cached per context (by the driver's context id): the first call in each
// context (the first call on a device, and again after cudaDeviceReset or in
// a context the caller created) does the lookup and should come before any
// CUDA stream capture.  All calls share the array and it keeps the last
// call's contents: the reduction slot and the flag are cleared at the start
// of every call, and two calls whose work overlaps on the GPU (different
// streams, no ordering) race on it.  Sizes beyond the maximum are rejected
// with AIRT_ERR_ARG.  Column indices are the caller's device data, which the
// host cannot inspect without a copy: an index outside [0, n) is skipped by
// the kernel and the call writes NaN to *d_resnorm.
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "spmv.cuh"

namespace airt {
namespace {

constexpr int64_t kNoAllocMaxN = int64_t(1) << 20;  // image pixels (1024 x 1024)
constexpr size_t kNoAllocBytes = (size_t)kNoAllocMaxN * sizeof(float) + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Scratch address per CUDA context, keyed by the driver's unique context id
// (a context created after a reset gets a new id even if it reuses a handle).
constexpr int kMaxContexts = 64;
struct ScratchSlot {
  unsigned long long ctx_id;
  unsigned char *addr;
};
std::mutex g_noalloc_mu;
ScratchSlot g_noalloc_slots[kMaxContexts];
int g_noalloc_nslots = 0;

// x (FP64) -> FP32 gather copy; one thread also clears the reduction slot
// and the bad-index flag.
__global__ void k_noalloc_prepare(int64_t n, const double *__restrict__ x, float *__restrict__ x32,
                                  double *__restrict__ acc, int *__restrict__ bad) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *acc = 0.0;
    *bad = 0;
  }
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x)
    x32[j] = (float)x[j];
}

// The forward residual of the SIRT iteration (k_sirt_fwd) without the
// M-weighting: r = b - A*x over the caller's FP32 CSR, ||r||^2 into *acc.
// One LANES-wide group per row, element-wise loads; a column index outside
// [0, n) is skipped and raises *bad.
template <int LANES>
__global__ void __launch_bounds__(256) k_noalloc_resid(int64_t m, int64_t n,
                                                       const int64_t *__restrict__ rp,
                                                       const int *__restrict__ ci,
                                                       const float *__restrict__ rv,
                                                       const float *__restrict__ x32,
                                                       const double *__restrict__ b,
                                                       double *__restrict__ r,
                                                       double *__restrict__ acc,
                                                       int *__restrict__ bad) {
  const int lane = threadIdx.x % LANES;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / LANES;
  const int64_t ng = (int64_t)gridDim.x * blockDim.x / LANES;
  const int64_t trips = (m + ng - 1) / ng;
  double a = 0.0;
  bool oob = false;
  for (int64_t t = 0; t < trips; ++t) {
    const int64_t i = gid + t * ng;
    double s = 0.0;
    if (i < m) {
      const int64_t q1 = rp[i + 1];
      for (int64_t q = rp[i] + lane; q < q1; q += LANES) {
        const int c = __ldg(ci + q);
        if (c >= 0 && c < n)
          s = fma((double)__ldg(rv + q), (double)x32[c], s);
        else
          oob = true;
      }
    }
    s = group_sum<LANES>(s);
    if (lane == 0 && i < m) {
      const double ri = b[i] - s;
      r[i] = ri;
      a += ri * ri;
    }
  }
  if (oob) atomicExch(bad, 1);
  a = block_sum<256>(a);
  if (threadIdx.x == 0) atomicAdd(acc, a);
}

__global__ void k_noalloc_finish(const double *__restrict__ acc, const int *__restrict__ bad,
                                 double *__restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *out = *bad ? __longlong_as_double(0x7ff8000000000000LL)
                                                      : sqrt(*acc);
}

using PFN_ctxGetCurrent = CUresult(CUDAAPI *)(CUcontext *);
using PFN_ctxGetId = CUresult(CUDAAPI *)(CUcontext, unsigned long long *);

// The current context's id, through the driver entry points the runtime
// hands out (the library does not link libcuda).  Makes the device's primary
// context current first when the calling thread has no context, as any
// runtime call would.
unsigned long long current_context_id() {
  static PFN_ctxGetCurrent get_current = nullptr;
  static PFN_ctxGetId get_id = nullptr;
  if (!get_current || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    AIRT_CHECK_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1));
    AIRT_CHECK_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2));
    AIRT_REQUIRE(q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess && f1 && f2,
                 "the CUDA driver does not provide cuCtxGetCurrent/cuCtxGetId");
    get_current = reinterpret_cast<PFN_ctxGetCurrent>(f1);
    get_id = reinterpret_cast<PFN_ctxGetId>(f2);
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) {
    int dev = 0;
    AIRT_CHECK_CUDA(cudaGetDevice(&dev));
    AIRT_CHECK_CUDA(cudaSetDevice(dev));   // binds the device's primary context
    ctx = nullptr;
    AIRT_REQUIRE(get_current(&ctx) == CUDA_SUCCESS && ctx, "no current CUDA context");
  }
  unsigned long long id = 0;
  AIRT_REQUIRE(get_id(ctx, &id) == CUDA_SUCCESS, "cuCtxGetId failed");
  return id;
}

unsigned char *scratch_address() {
  const unsigned long long id = current_context_id();
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  for (int k = 0; k < g_noalloc_nslots; ++k)
    if (g_noalloc_slots[k].ctx_id == id) return g_noalloc_slots[k].addr;
  void *p = nullptr;
  AIRT_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
  // contexts beyond the table's size are looked up on every call
  if (g_noalloc_nslots < kMaxContexts)
    g_noalloc_slots[g_noalloc_nslots++] = ScratchSlot{id, static_cast<unsigned char *>(p)};
  return static_cast<unsigned char *>(p);
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
    int *bad = reinterpret_cast<int *>(base + (size_t)kNoAllocMaxN * sizeof(float) + 8);
    k_noalloc_prepare<<<grid_for(n > 0 ? n : 1, 256), 256, 0, s>>>(n, d_x, x32, acc, bad);
    AIRT_LAUNCH_CHECK();
    if (m > 0) {
      k_noalloc_resid<8><<<grid_for(m * 8, 256), 256, 0, s>>>(m, n, d_rp, d_ci, d_rv, x32, d_b,
                                                              d_r, acc, bad);
      AIRT_LAUNCH_CHECK();
    }
    k_noalloc_finish<<<1, 32, 0, s>>>(acc, bad, d_resnorm);
    AIRT_LAUNCH_CHECK();
  } catch (const Status &st) {
    return st.code;
  } catch (...) {
    set_error("unexpected internal error");
    return AIRT_ERR_CUDA;
  }
  return AIRT_OK;
}
