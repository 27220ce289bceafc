// noalloc.cu -- CFL time-step reduction for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is owned by
// an external pool (the pool hands out every byte, and a stray allocation would
// break its accounting or fail), and time-critical loops that cannot afford the
// implicit synchronisation an allocation can bring.  storm_fvt_cfl_dt_noalloc gives them the same CFL time step that
// storm_fvt_step computes for dt_op = 1 without allocating anything: its scratch
// (one FP64 partial minimum per thread block) lives in the file-scope array below,
// which every GPU that loads this library holds (32 KiB) until the process exits.
//
// Limits and rules of use:
//   * at most kNoAllocMaxCells cells per call (4,096 blocks x 256 threads); larger
//     inputs are rejected with STORM_ERR_ARG before anything is launched;
//   * the array's address belongs to a CUDA context, not to a device ordinal.  A call
//     made outside stream capture resolves it with cudaGetSymbolAddress in the
//     calling thread's current context and records it for that context; a call made
//     while `stream` is being captured uses the recorded address of the current
//     context and fails (STORM_ERR_ARG) if that context has none;
//   * with CUDA's lazy module loading, the first call in a context loads this
//     library's device module, and loading it allocates device memory for the array
//     and the code and may synchronise.  Make that first call while allocation is
//     still allowed: before an external pool takes the device's memory, and outside
//     any stream capture.  After cudaDeviceReset, or when a context is destroyed and
//     another made current, make one call outside capture again before capturing;
//   * every call shares the one array, which keeps the last call's partials; a call
//     overwrites every partial it reads, so nothing needs clearing, but calls that
//     overlap on the GPU (different streams, or different host threads) race;
//   * the call is asynchronous on `stream`: *d_dt is valid once the stream reaches it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "storm_internal.h"

namespace storm {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaMaxBlocks = 4096;
constexpr int64_t kNoAllocMaxCells = (int64_t)kNaMaxBlocks * kNaThreads;  // 1,048,576

static __device__ __align__(256) double g_dt_partials[kNaMaxBlocks];

constexpr double kG = 9.81;
constexpr double kFmachp = 2.220446049250313e-16;
constexpr double kVsmall = 2.2250738585072014e-308;
constexpr double kVlarge = 1.7976931348623157e+308;
#define NA_SMALL ((double)1.0e-9f)

__device__ __forceinline__ double na_min(double a, double b) { return (b < a) ? b : a; }

// The per-cell CFL candidate of k_fric: find_dry_cells (find_dry_cells.f90:25-42),
// wavec (solverFVT.f90:180-181) and cfl*area/((|u|+c+small)*perim) (deltatFVT.f90:34-37
// with the cell area and perimeter).
__global__ void __launch_bounds__(kNaThreads)
    k_cfl_dt_partials(const double* __restrict__ h, const double* __restrict__ u, const double* __restrict__ v,
                      const double* __restrict__ area, const double* __restrict__ perim, int n, double cfl,
                      double h_dry, double h_wet, double* __restrict__ part) {
  __shared__ double sm[kNaThreads / 32];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double cand = kVlarge;
  if (c < n) {
    const double hh = h[c], uu = u[c], vv = v[c];
    bool dry = hh < h_dry;
    double um = 0.0;
    if (!dry) um = sqrt(uu * uu + vv * vv);
    if (!dry && (hh < h_wet)) {
      double eps = fabs(um) * kFmachp;
      if (eps == 0.0) eps = kVsmall;
      if (!(fabs(um - 0.0) > eps)) dry = true;
    }
    const double wc = dry ? 0.0 : sqrt(kG * hh);
    cand = cfl * area[c] / ((um + wc + NA_SMALL) * perim[c]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cand = na_min(cand, __shfl_xor_sync(0xffffffffu, cand, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = cand;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = sm[0];
    for (int i = 1; i < kNaThreads / 32; i++) r = na_min(r, sm[i]);
    part[blockIdx.x] = r;
  }
}

__global__ void __launch_bounds__(kNaThreads) k_cfl_dt_final(const double* __restrict__ part, int nblk,
                                                             double* __restrict__ out) {
  __shared__ double sm[kNaThreads / 32];
  double m = kVlarge;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) m = na_min(m, part[b]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = na_min(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = sm[0];
    for (int i = 1; i < kNaThreads / 32; i++) r = na_min(r, sm[i]);
    *out = r;
  }
}

// Address of g_dt_partials per CUDA context (the driver's CUcontext handle), looked up
// through the runtime's driver entry point so the library needs no link to libcuda.
using CtxGetCurrentFn = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)
std::mutex g_na_mutex;
CtxGetCurrentFn g_ctx_get = nullptr;
std::vector<std::pair<void*, double*>> g_na_addr;

int current_context(void** ctx) {
  if (!g_ctx_get) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return set_error(STORM_ERR_CUDA, "storm_fvt_cfl_dt_noalloc: cuCtxGetCurrent is not available");
    g_ctx_get = reinterpret_cast<CtxGetCurrentFn>(fn);
  }
  *ctx = nullptr;
  if (g_ctx_get(ctx) != 0) return set_error(STORM_ERR_CUDA, "storm_fvt_cfl_dt_noalloc: cuCtxGetCurrent failed");
  return STORM_OK;
}

}  // namespace
}  // namespace storm

extern "C" int storm_fvt_cfl_dt_noalloc(const double* d_h, const double* d_u, const double* d_v,
                                        const double* d_area, const double* d_perim, int32_t n, double cfl,
                                        double h_dry, double h_wet, double* d_dt, void* stream) {
  using namespace storm;
  clear_error();
  if (!d_h || !d_u || !d_v || !d_area || !d_perim || !d_dt)
    return set_error(STORM_ERR_ARG, "storm_fvt_cfl_dt_noalloc: null pointer");
  if (n < 1) return set_error(STORM_ERR_ARG, "storm_fvt_cfl_dt_noalloc: n must be at least 1");
  if ((int64_t)n > kNoAllocMaxCells)
    return set_error(STORM_ERR_ARG, "storm_fvt_cfl_dt_noalloc: n = " + std::to_string(n) +
                                        " exceeds the static scratch limit of " +
                                        std::to_string(kNoAllocMaxCells) + " cells");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess)
    return set_error(STORM_ERR_CUDA, std::string("storm_fvt_cfl_dt_noalloc: ") + cudaGetErrorString(e));
  double* part = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    void* ctx = nullptr;
    if (cap == cudaStreamCaptureStatusNone) {
      // resolve in the current context (this also makes the primary context current
      // on a thread that has none yet), then record it for that context
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_dt_partials);
      if (e != cudaSuccess || !p)
        return set_error(STORM_ERR_CUDA, std::string("storm_fvt_cfl_dt_noalloc: cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
      int rc = current_context(&ctx);
      if (rc) return rc;
      part = static_cast<double*>(p);
      bool found = false;
      for (auto& kv : g_na_addr)
        if (kv.first == ctx) {
          kv.second = part;
          found = true;
        }
      if (!found) g_na_addr.emplace_back(ctx, part);
    } else {
      int rc = current_context(&ctx);
      if (rc) return rc;
      for (const auto& kv : g_na_addr)
        if (kv.first == ctx) part = kv.second;
      if (!part)
        return set_error(STORM_ERR_ARG,
                         "storm_fvt_cfl_dt_noalloc: first call in this CUDA context made during stream capture; "
                         "make one call outside capture first");
    }
  }
  const int nblk = (n + kNaThreads - 1) / kNaThreads;
  k_cfl_dt_partials<<<nblk, kNaThreads, 0, s>>>(d_h, d_u, d_v, d_area, d_perim, n, cfl, h_dry, h_wet, part);
  k_cfl_dt_final<<<1, kNaThreads, 0, s>>>(part, nblk, d_dt);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_error(STORM_ERR_CUDA, std::string("storm_fvt_cfl_dt_noalloc: launch: ") + cudaGetErrorString(e));
  return STORM_OK;
}
