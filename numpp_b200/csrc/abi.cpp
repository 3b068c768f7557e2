// extern "C" entry points for uniform batches and the GpuVTable slots.
// C++20 host code over the sm_100a kernels; no exception crosses the ABI.
#include <cuda_runtime.h>

#include <climits>
#include <cstring>
#include <new>
#include <string>

#include "../../include/numpp_b200.h"
#include "plan.hpp"
#include "runtime.hpp"

using namespace nppb;

namespace {

template <class F>
int guarded(F&& f) {
  try {
    clear_error();
    return f();
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return NPPB_E_NOMEM;
  } catch (const std::exception& e) {
    set_error(e.what());
    return NPPB_E_ARG;
  }
}

int arg_error(const char* msg) {
  set_error(msg);
  return NPPB_E_ARG;
}

// count/n/nrhs checks shared by every batched entry point.
int check_shape(int64_t count, int32_t n, int32_t nrhs) {
  if (count < 0 || n < 0 || nrhs < 0) return arg_error("negative count, order or nrhs");
  if (count > INT_MAX) {
    set_error("batch count above 2^31-1");
    return NPPB_E_RANGE;
  }
  if (n > kStepMaxN) {
    set_error("order above " + std::to_string(kStepMaxN) + " is not served by the batched path");
    return NPPB_E_RANGE;
  }
  return NPPB_OK;
}

#define NPPB_CUDA(call, what)                   \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_status(e_, what); \
  } while (0)

// Host <-> device staging for the host-buffer entry points.
template <class T>
int upload(DevMem& m, const T* h, size_t n, cudaStream_t st) {
  NPPB_CUDA(m.alloc(n * sizeof(T), st), "device allocation");
  if (n) NPPB_CUDA(cudaMemcpyAsync(m.as<T>(), h, n * sizeof(T), cudaMemcpyHostToDevice, st), "host to device copy");
  return NPPB_OK;
}
template <class T>
int scratch(DevMem& m, size_t n, cudaStream_t st) {
  NPPB_CUDA(m.alloc(n * sizeof(T), st), "device allocation");
  return NPPB_OK;
}
template <class T>
int download(T* h, const DevMem& m, size_t n, cudaStream_t st) {
  if (n) NPPB_CUDA(cudaMemcpyAsync(h, m.as<T>(), n * sizeof(T), cudaMemcpyDeviceToHost, st), "device to host copy");
  return NPPB_OK;
}
int finish(cudaStream_t st) {
  NPPB_CUDA(cudaStreamSynchronize(st), "stream synchronize");
  NPPB_CUDA(cudaGetLastError(), "kernel");
  return NPPB_OK;
}

#define NPPB_RC(expr)          \
  do {                         \
    int rc_ = (expr);          \
    if (rc_ != NPPB_OK) return rc_; \
  } while (0)

int d_linalg(int64_t count, int32_t n, int32_t nrhs, int flags, const double* dA, const double* dB,
             double* dX, double* dInv, double* dDet, double* dSign, double* dLogabs, double* dLU,
             int32_t* dipiv, int32_t* dinfo, cudaStream_t st) {
  NPPB_RC(check_shape(count, n, nrhs));
  if (flags & ~(NPPB_WANT_LU | NPPB_WANT_SOLVE | NPPB_WANT_DET | NPPB_WANT_SLOGDET | NPPB_WANT_INV))
    return arg_error("unknown flag bits");
  if (count == 0) return NPPB_OK;
  const size_t nn = (size_t)n * n;
  if (!dA && nn) return arg_error("A is null");
  if ((flags & NPPB_WANT_SOLVE) && nrhs && (!dB || !dX)) return arg_error("solve needs B and X");
  if ((flags & NPPB_WANT_INV) && nn && !dInv) return arg_error("inverse needs Inv");
  if ((flags & NPPB_WANT_DET) && !dDet) return arg_error("det needs Det");
  if ((flags & NPPB_WANT_SLOGDET) && (!dSign || !dLogabs)) return arg_error("slogdet needs Sign and Logabs");
  if ((flags & NPPB_WANT_LU) && nn && (!dLU || !dipiv)) return arg_error("keeping factors needs LU and ipiv");
  if (!device()) return NPPB_E_NODEV;
  if (n > 32 && !(flags & NPPB_WANT_LU)) {
    // step-wise kernels in uniform mode: workspace and per-system scratch only
    DevMem lu_m, sc_m;
    double* LU = dLU;
    if (!LU) {
      NPPB_RC(scratch<double>(lu_m, (size_t)count * nn, st));
      LU = lu_m.as<double>();
    }
    NPPB_RC(scratch<StepScratch>(sc_m, (size_t)count, st));
    StepArgs sa{};
    sa.scratch = sc_m.as<StepScratch>();
    DevMem hist_m;
    const int bmin = blocked_min_n();
    if (bmin > 0 && n >= bmin) {  // two-level factorisation: per-system record of a block's panels
      NPPB_RC(scratch<StepHist>(hist_m, (size_t)count, st));
      sa.hist = hist_m.as<StepHist>();
    }
    sa.A = (dA == LU) ? nullptr : dA;
    sa.LU = LU;
    sa.ipiv = dipiv;
    sa.B = dB; sa.X = dX;
    sa.inv = (flags & NPPB_WANT_INV) ? dInv : nullptr;
    sa.det = (flags & NPPB_WANT_DET) ? dDet : nullptr;
    sa.sign = (flags & NPPB_WANT_SLOGDET) ? dSign : nullptr;
    sa.logabs = (flags & NPPB_WANT_SLOGDET) ? dLogabs : nullptr;
    sa.info = dinfo;
    sa.un = n;
    sa.unrhs = (flags & NPPB_WANT_SOLVE) ? nrhs : 0;
    sa.uinv = (flags & NPPB_WANT_INV) ? 1 : 0;
    NPPB_CUDA(run_step_uniform(sa, (int)count, st), "batched LU launch");
    return NPPB_OK;
  }
  if (n > 32) {
    // factors kept (getrf): a cached uniform plan also carries the row moves
    // into the columns left of each panel
    int rc = NPPB_OK;
    const bool own_lu = dLU == nullptr;
    auto pl = uniform_plan(count, n, nrhs, flags, false, own_lu, &rc);
    if (!pl) return rc;
    Plan::Ptrs p{};
    p.A = (dLU && dA == dLU) ? nullptr : dA;
    p.B = dB; p.X = dX; p.Inv = dInv; p.Det = dDet; p.Sign = dSign; p.Logabs = dLogabs;
    p.info = dinfo;
    p.LU = own_lu ? pl->d_lu : dLU;
    p.ipiv = dipiv ? dipiv : pl->d_piv;
    return pl->execute(p, st);
  }
  // the warp kernel writes factors and pivots only when they are kept: no
  // workspace otherwise (a small batch is then one launch and nothing else)
  DevMem lu_m, piv_m;
  double* LU = dLU;
  int32_t* piv = dipiv;
  if (flags & NPPB_WANT_LU) {
    if (!LU) {
      NPPB_RC(scratch<double>(lu_m, (size_t)count * nn, st));
      LU = lu_m.as<double>();
    }
    if (!piv) {
      NPPB_RC(scratch<int32_t>(piv_m, (size_t)count * n, st));
      piv = piv_m.as<int32_t>();
    }
  }
  Batch bt{};
  bt.A = dA; bt.LU = LU; bt.ipiv = piv; bt.B = dB; bt.X = dX;
  bt.inv = (flags & NPPB_WANT_INV) ? dInv : nullptr;
  bt.det = dDet; bt.sign = dSign; bt.logabs = dLogabs; bt.info = dinfo;
  bt.desc = nullptr; bt.n = n; bt.nrhs = nrhs;
  bt.flags = flags | (dA == LU ? kInPlace : 0);
  NPPB_CUDA(run_warp_uniform(bt, count, n, st), "batched LU launch");
  return NPPB_OK;
}

int d_getrs(int64_t count, int32_t n, int32_t nrhs, const double* dLU, const int32_t* dipiv,
            const double* dB, double* dX, cudaStream_t st) {
  NPPB_RC(check_shape(count, n, nrhs));
  if (count == 0 || n == 0 || nrhs == 0) return NPPB_OK;
  if (!dLU || !dipiv || !dB || !dX) return arg_error("getrs needs LU, ipiv, B and X");
  if (!device()) return NPPB_E_NODEV;
  if (n > 32) {
    int rc = NPPB_OK;
    auto pl = uniform_plan(count, n, nrhs, NPPB_WANT_SOLVE, true, false, &rc);
    if (!pl) return rc;
    DevMem tmp;
    double* X = dX;
    if (dX == dB) {  // the row gather needs a separate output
      NPPB_RC(scratch<double>(tmp, (size_t)count * n * nrhs, st));
      X = tmp.as<double>();
    }
    Plan::Ptrs p{};
    p.B = dB; p.X = X;
    p.LU = const_cast<double*>(dLU);
    p.ipiv = const_cast<int32_t*>(dipiv);
    NPPB_RC(pl->execute(p, st));
    if (X != dX)
      NPPB_CUDA(cudaMemcpyAsync(dX, X, sizeof(double) * count * n * nrhs, cudaMemcpyDeviceToDevice, st),
                "device copy");
    return NPPB_OK;
  }
  Batch bt{};
  bt.A = dLU; bt.LU = const_cast<double*>(dLU); bt.ipiv = const_cast<int32_t*>(dipiv);
  bt.B = dB; bt.X = dX; bt.n = n; bt.nrhs = nrhs;
  bt.flags = kSolveOnly | kWantSolve | kInPlace;
  NPPB_CUDA(run_warp_uniform(bt, count, n, st), "getrs launch");
  return NPPB_OK;
}

// Host-buffer batched call: stage inputs, run, copy the requested outputs back.
int h_linalg(int64_t count, int32_t n, int32_t nrhs, int flags, const double* A, const double* B,
             double* X, double* Inv, double* Det, double* Sign, double* Logabs, int32_t* info) {
  NPPB_RC(check_shape(count, n, nrhs));
  if (count == 0) return NPPB_OK;
  if (!device()) return NPPB_E_NODEV;
  cudaStream_t st = thread_stream();
  const size_t nn = (size_t)count * n * n, nb = (size_t)count * n * nrhs, c = (size_t)count;
  const bool solve = (flags & NPPB_WANT_SOLVE) && nb;
  if (nn && !A) return arg_error("A is null");
  if (solve && (!B || !X)) return arg_error("solve needs B and X");
  DevMem dA, dB, dX, dInv, dDet, dSign, dLog, dInfo;
  NPPB_RC(upload(dA, A, nn, st));
  if (solve) {
    NPPB_RC(upload(dB, B, nb, st));
    NPPB_RC(scratch<double>(dX, nb, st));
  }
  if (flags & NPPB_WANT_INV) NPPB_RC(scratch<double>(dInv, nn, st));
  if (flags & NPPB_WANT_DET) NPPB_RC(scratch<double>(dDet, c, st));
  if (flags & NPPB_WANT_SLOGDET) {
    NPPB_RC(scratch<double>(dSign, c, st));
    NPPB_RC(scratch<double>(dLog, c, st));
  }
  NPPB_RC(scratch<int32_t>(dInfo, c, st));
  NPPB_RC(d_linalg(count, n, nrhs, flags & ~NPPB_WANT_LU, dA.as<double>(), dB.as<double>(),
                   dX.as<double>(), dInv.as<double>(), dDet.as<double>(), dSign.as<double>(),
                   dLog.as<double>(), nullptr, nullptr, dInfo.as<int32_t>(), st));
  if (solve) NPPB_RC(download(X, dX, nb, st));
  if (flags & NPPB_WANT_INV) NPPB_RC(download(Inv, dInv, nn, st));
  if (flags & NPPB_WANT_DET) NPPB_RC(download(Det, dDet, c, st));
  if (flags & NPPB_WANT_SLOGDET) {
    NPPB_RC(download(Sign, dSign, c, st));
    NPPB_RC(download(Logabs, dLog, c, st));
  }
  if (info) NPPB_RC(download(info, dInfo, c, st));
  return finish(st);
}

}  // namespace

extern "C" {

int nppb_abi_version(void) { return NPPB_ABI_VERSION; }

int nppb_device_available(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess || c == 0) {
    cudaGetLastError();
    return 0;
  }
  return device() ? 1 : 0;
}

const char* nppb_last_error(void) { return last_error(); }

int32_t nppb_max_order(void) { return kStepMaxN; }

int nppb_elementwise_binary(int, int, int64_t, const void*, const void*, void*) { return NPPB_DECLINED; }
int nppb_elementwise_unary(int, int, int64_t, const void*, void*) { return NPPB_DECLINED; }
int nppb_reduce(int, int, int64_t, const void*, void*) { return NPPB_DECLINED; }

int nppb_d_gemm(int dtype, int64_t m, int64_t n, int64_t k, const void* dA, const void* dB, void* dC,
                void* stream) {
  return guarded([&]() -> int {
    if (dtype != NPPB_DT_FLOAT64 && dtype != NPPB_DT_FLOAT32) return NPPB_DECLINED;
    if (m < 0 || n < 0 || k < 0) return arg_error("negative GEMM extent");
    if (m == 0 || n == 0) return NPPB_OK;
    if ((k && (!dA || !dB)) || !dC) return arg_error("null GEMM operand");
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dtype == NPPB_DT_FLOAT64)
      NPPB_CUDA(launch_gemm_f64(m, n, k, (const double*)dA, k, (const double*)dB, n, (double*)dC, n, st),
                "gemm launch");
    else
      NPPB_CUDA(launch_gemm_f32(m, n, k, (const float*)dA, (const float*)dB, (float*)dC, st), "gemm launch");
    return NPPB_OK;
  });
}

int nppb_gemm(int dtype, int64_t m, int64_t n, int64_t k, const void* A, const void* B, void* C) {
  return guarded([&]() -> int {
    if (dtype != NPPB_DT_FLOAT64 && dtype != NPPB_DT_FLOAT32) return NPPB_DECLINED;
    if (m < 0 || n < 0 || k < 0) return arg_error("negative GEMM extent");
    if (m == 0 || n == 0) return NPPB_OK;
    if (!device()) return NPPB_E_NODEV;
    const size_t es = dtype == NPPB_DT_FLOAT64 ? 8 : 4;
    cudaStream_t st = thread_stream();
    DevMem dA, dB, dC;
    NPPB_RC(upload(dA, (const char*)A, (size_t)m * k * es, st));
    NPPB_RC(upload(dB, (const char*)B, (size_t)k * n * es, st));
    NPPB_RC(scratch<char>(dC, (size_t)m * n * es, st));
    NPPB_RC(nppb_d_gemm(dtype, m, n, k, dA.as<void>(), dB.as<void>(), dC.as<void>(), st));
    NPPB_RC(download((char*)C, dC, (size_t)m * n * es, st));
    return finish(st);
  });
}

int nppb_d_linalg_batched(int64_t count, int32_t n, int32_t nrhs, int flags, const double* dA,
                          const double* dB, double* dX, double* dInv, double* dDet, double* dSign,
                          double* dLogabs, double* dLU, int32_t* dipiv, int32_t* dinfo, void* stream) {
  return guarded([&]() -> int {
    return d_linalg(count, n, nrhs, flags, dA, dB, dX, dInv, dDet, dSign, dLogabs, dLU, dipiv, dinfo,
                    static_cast<cudaStream_t>(stream));
  });
}

int nppb_d_getrs_batched(int64_t count, int32_t n, int32_t nrhs, const double* dLU,
                         const int32_t* dipiv, const double* dB, double* dX, void* stream) {
  return guarded([&]() -> int {
    return d_getrs(count, n, nrhs, dLU, dipiv, dB, dX, static_cast<cudaStream_t>(stream));
  });
}

int nppb_getrf_batched(int64_t count, int32_t n, double* A, int32_t* ipiv, int32_t* info) {
  return guarded([&]() -> int {
    NPPB_RC(check_shape(count, n, 0));
    if (count == 0) return NPPB_OK;
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t nn = (size_t)count * n * n, np = (size_t)count * n;
    if ((nn && (!A || !ipiv)) || !info) return arg_error("getrf needs A, ipiv and info");
    DevMem dA, dP, dI;
    NPPB_RC(upload(dA, A, nn, st));
    NPPB_RC(scratch<int32_t>(dP, np, st));
    NPPB_RC(scratch<int32_t>(dI, count, st));
    NPPB_RC(d_linalg(count, n, 0, NPPB_WANT_LU, dA.as<double>(), nullptr, nullptr, nullptr, nullptr,
                     nullptr, nullptr, dA.as<double>(), dP.as<int32_t>(), dI.as<int32_t>(), st));
    NPPB_RC(download(A, dA, nn, st));
    NPPB_RC(download(ipiv, dP, np, st));
    NPPB_RC(download(info, dI, count, st));
    return finish(st);
  });
}

int nppb_getrs_batched(int64_t count, int32_t n, int32_t nrhs, const double* LU, const int32_t* ipiv,
                       double* B) {
  return guarded([&]() -> int {
    NPPB_RC(check_shape(count, n, nrhs));
    if (count == 0 || n == 0 || nrhs == 0) return NPPB_OK;
    if (!LU || !ipiv || !B) return arg_error("getrs needs LU, ipiv and B");
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t nn = (size_t)count * n * n, np = (size_t)count * n, nb = (size_t)count * n * nrhs;
    DevMem dL, dP, dB;
    NPPB_RC(upload(dL, LU, nn, st));
    NPPB_RC(upload(dP, ipiv, np, st));
    NPPB_RC(upload(dB, B, nb, st));
    NPPB_RC(d_getrs(count, n, nrhs, dL.as<double>(), dP.as<int32_t>(), dB.as<double>(), dB.as<double>(), st));
    NPPB_RC(download(B, dB, nb, st));
    return finish(st);
  });
}

int nppb_solve_batched(int64_t count, int32_t n, int32_t nrhs, const double* A, const double* B,
                       double* X, int32_t* info) {
  return guarded([&]() -> int {
    return h_linalg(count, n, nrhs, NPPB_WANT_SOLVE, A, B, X, nullptr, nullptr, nullptr, nullptr, info);
  });
}

int nppb_inv_batched(int64_t count, int32_t n, const double* A, double* Ainv, int32_t* info) {
  return guarded([&]() -> int {
    if (count > 0 && n > 0 && !Ainv) return arg_error("Ainv is null");
    return h_linalg(count, n, 0, NPPB_WANT_INV, A, nullptr, nullptr, Ainv, nullptr, nullptr, nullptr, info);
  });
}

int nppb_det_batched(int64_t count, int32_t n, const double* A, double* det) {
  return guarded([&]() -> int {
    if (count > 0 && !det) return arg_error("det is null");
    return h_linalg(count, n, 0, NPPB_WANT_DET, A, nullptr, nullptr, nullptr, det, nullptr, nullptr, nullptr);
  });
}

int nppb_slogdet_batched(int64_t count, int32_t n, const double* A, double* sign, double* logabsdet) {
  return guarded([&]() -> int {
    if (count > 0 && (!sign || !logabsdet)) return arg_error("sign/logabsdet is null");
    return h_linalg(count, n, 0, NPPB_WANT_SLOGDET, A, nullptr, nullptr, nullptr, nullptr, sign, logabsdet,
                    nullptr);
  });
}

int nppb_solve_det_batched(int64_t count, int32_t n, int32_t nrhs, const double* A, const double* B,
                           double* X, double* det, int32_t* info) {
  return guarded([&]() -> int {
    if (count > 0 && !det) return arg_error("det is null");
    return h_linalg(count, n, nrhs, NPPB_WANT_SOLVE | NPPB_WANT_DET, A, B, X, nullptr, det, nullptr,
                    nullptr, info);
  });
}

}  // extern "C"
