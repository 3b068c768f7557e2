// Allocation-free batched solve: nppb_d_solve_batched_noalloc.
//
// For callers that cannot allocate device memory while they run: real-time or
// embedded hosts that reserve all device memory up front, and fixed-pool
// allocators where a cudaMalloc would fail or stall mid-run. The solve of a
// uniform batch needs an LU workspace and per-system step state for orders
// above 32; here they live in one file-scope device array of fixed size
// instead of being allocated per call. The array belongs to the library's
// module, so its 32 MiB are reserved on every device where that module is
// loaded (each context under eager module loading; the first use under lazy
// loading) until the process exits.
//
// The array is a host-side symbol in host code, not a device address: its
// device address is fetched once per device with cudaGetSymbolAddress (the
// first call on each device does that, with the device current, so make that
// first call before any stream capture) and only that address is passed to
// the kernels. Every call shares the array and it keeps the last call's
// contents; nothing in it needs to start at zero (every call writes the LU
// workspace and the step state before reading them). Calls that overlap on the
// GPU race on it.
//
// This solve always takes the single-level step kernels (it ignores
// NPPB_BLOCKED_MIN_N, whose two-level schedule needs a per-call history
// buffer), so with that variable set its results can differ from the
// allocating solve's in the last bits.
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <new>
#include <string>

#include "../../include/numpp_b200.h"
#include "nppb_step.hpp"
#include "runtime.hpp"

namespace nppb {
namespace {

constexpr size_t kNoAllocBytes = size_t(32) << 20;  // 32 MiB on every device that loads the module

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal out of range for the scratch table");
    return NPPB_E_RANGE;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(scratch)");
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return NPPB_OK;
}

}  // namespace
}  // namespace nppb

using namespace nppb;

namespace {

int solve_noalloc(int64_t count, int32_t n, int32_t nrhs, const double* dA, const double* dB, double* dX,
                  int32_t* dinfo, void* stream) {
  if (count < 0 || n < 0 || nrhs < 0) {
    set_error("negative count, order or nrhs");
    return NPPB_E_ARG;
  }
  if (n > kStepMaxN || count > INT32_MAX) {
    set_error("order above " + std::to_string(kStepMaxN) + " or count above 2^31-1");
    return NPPB_E_RANGE;
  }
  const size_t lu_bytes = ((size_t)count * n * n * sizeof(double) + 255) / 256 * 256;
  const size_t need = n > 32 ? lu_bytes + (size_t)count * sizeof(StepScratch) : 0;
  if (need > kNoAllocBytes) {
    set_error("batch needs " + std::to_string(need) + " bytes of scratch; the allocation-free solve holds " +
              std::to_string(kNoAllocBytes) + " (count * (8*n*n + " + std::to_string(sizeof(StepScratch)) +
              ") for n > 32)");
    return NPPB_E_RANGE;
  }
  if (count == 0) return NPPB_OK;
  if ((n && (!dA || (nrhs && (!dB || !dX)))) || !dinfo) {
    set_error("A, B, X and info are required");
    return NPPB_E_ARG;
  }
  if (!device()) return NPPB_E_NODEV;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (n <= 32) {
    // the warp kernel keeps everything in registers: no scratch at all
    Batch bt{};
    bt.A = dA;
    bt.LU = const_cast<double*>(dA);  // not written without kWantLU
    bt.B = dB;
    bt.X = dX;
    bt.info = dinfo;
    bt.n = n;
    bt.nrhs = nrhs;
    bt.flags = kWantSolve;
    e = run_warp_uniform(bt, count, n, st);
  } else {
    void* base = nullptr;
    const int rc = scratch_address(&base);
    if (rc != NPPB_OK) return rc;
    StepArgs sa{};
    sa.LU = static_cast<double*>(base);
    sa.scratch = reinterpret_cast<StepScratch*>(static_cast<unsigned char*>(base) + lu_bytes);
    sa.A = dA;
    sa.B = dB;
    sa.X = dX;
    sa.info = dinfo;
    sa.un = n;
    sa.unrhs = nrhs;
    sa.uinv = 0;
    e = run_step_uniform(sa, (int)count, st);
  }
  if (e != cudaSuccess) return cuda_status(e, "allocation-free solve launch");
  return NPPB_OK;
}

}  // namespace

extern "C" int nppb_d_solve_batched_noalloc(int64_t count, int32_t n, int32_t nrhs, const double* dA,
                                            const double* dB, double* dX, int32_t* dinfo,
                                            void* stream) {
  try {  // error text is a std::string: no exception may leave the C ABI
    clear_error();
    return solve_noalloc(count, n, nrhs, dA, dB, dX, dinfo, stream);
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return NPPB_E_NOMEM;
  }
}
