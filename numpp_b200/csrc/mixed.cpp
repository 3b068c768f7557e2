// Mixed-precision batched solve: FP32 factors, FP64 iterative refinement. C++20.
//
// No counterpart in the reference (NumPP solves in double only,
// src/linalg/linalg.cpp:92-103). For a uniform batch of order n:
//  1. equilibrate: power-of-two row/column scales;
//  2. factor in FP32. Default: the scaled matrix mixed by random butterflies
//     on both sides and factored in 128-column blocks with pivoting inside
//     each diagonal block, every block's triangular solves and trailing update
//     as tcgen05 GEMMs with error-compensated TF32 products (k_mxlu.cu). With
//     a pivoted flag: partial pivoting on the step-wise kernels (row moves
//     kept), the first solution riding along as augmented columns, trailing
//     products as error-compensated TF32, TF32, BF16 (mma.sync or tcgen05) or
//     FP32 FMA;
//  3. refine in FP64: R = B - A X, eta = normwise backward error; systems with
//     eta <= tol stop, systems whose contraction cannot reach tol are marked
//     stalled; the others solve A d = R with the FP32 factors and add d in
//     FP64 (with NPPB_MIXED_GMRES: d by GMRES on M^-1 A d = M^-1 R, M the FP32
//     factorisation applied to FP64 vectors, Carson and Higham's GMRES-IR);
//  4. every system that did not converge (stalled, FP32 zero pivot, or out of
//     iterations) is refactored and solved in FP64;
//  5. report per system: eta, forward error when X_true is given, corrections
//     applied, and whether the FP64 fallback ran.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "../../include/numpp_b200.h"
#include "gmres.hpp"
#include "mixed.hpp"
#include "mxlu.hpp"
#include "runtime.hpp"

using namespace nppb;

namespace {

// relative residual at which GMRES stops inside one correction (the outer
// FP64 residual decides convergence)
constexpr double kGmresTau = 1e-6;

#define NPPB_CUDA(call, what)                            \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_status(e_, what); \
  } while (0)
#define NPPB_RC(expr)               \
  do {                              \
    int rc_ = (expr);               \
    if (rc_ != NPPB_OK) return rc_; \
  } while (0)

int mixed(int64_t count64, int32_t n, int32_t nrhs, const double* dA, const double* dB, double* dX,
          const double* dXtrue, double tol, int32_t max_iter, int flags, int32_t* dinfo, double* dBerr,
          double* dFerr, int32_t* dIters, int32_t* dFallback, cudaStream_t st) {
  if (count64 < 0 || n < 0 || nrhs < 0 || max_iter < 0 || !(tol >= 0.0)) {
    set_error("negative count, order, nrhs or max_iter, or bad tolerance");
    return NPPB_E_ARG;
  }
  const int arith = flags & (NPPB_MIXED_TF32 | NPPB_MIXED_BF16 | NPPB_MIXED_FP32_FMA);
  if ((flags & ~(NPPB_MIXED_NO_EQUILIBRATE | NPPB_MIXED_NO_FALLBACK | NPPB_MIXED_TF32 | NPPB_MIXED_BF16 |
                 NPPB_MIXED_FP32_FMA | NPPB_MIXED_TCGEN05 | NPPB_MIXED_PIVOTED | NPPB_MIXED_GMRES)) ||
      (arith & (arith - 1))) {
    set_error("unknown mixed flag bits, or more than one of TF32 / BF16 / FP32_FMA");
    return NPPB_E_ARG;
  }
  if (n > kMixedMaxN || count64 > INT32_MAX) {
    set_error("order above " + std::to_string(kMixedMaxN) + " or count above 2^31-1");
    return NPPB_E_RANGE;
  }
  if (count64 == 0 || n == 0 || nrhs == 0) return NPPB_OK;
  if (!dA || !dB || !dX) {
    set_error("A, B and X are required");
    return NPPB_E_ARG;
  }
  if (!device()) return NPPB_E_NODEV;
  const int count = (int)count64;
  const size_t nn = (size_t)n * n, nb = (size_t)n * nrhs, c = (size_t)count;
  const bool pivoted =
      (flags & (NPPB_MIXED_PIVOTED | NPPB_MIXED_TF32 | NPPB_MIXED_BF16 | NPPB_MIXED_FP32_FMA | NPPB_MIXED_TCGEN05)) != 0;
  const bool blocked = n > 32 && !pivoted;
  const bool gmres = blocked && (flags & NPPB_MIXED_GMRES);
  if ((flags & NPPB_MIXED_GMRES) && pivoted) {
    set_error("GMRES refinement runs on the default (blocked) factorisation only");
    return NPPB_E_ARG;
  }
  DevMem a32, piv, rpos, sc32, b32, y32, rsm, csm, cmx, stm, info32, act, mxw;
  if (!blocked) {
    NPPB_CUDA(a32.alloc(sizeof(float) * c * nn, st), "workspace");
    NPPB_CUDA(piv.alloc(sizeof(int32_t) * c * n, st), "workspace");
    NPPB_CUDA(rpos.alloc(sizeof(int32_t) * c * n, st), "workspace");
    NPPB_CUDA(sc32.alloc(sizeof(StepScratchT<float>) * c, st), "workspace");
    NPPB_CUDA(y32.alloc(sizeof(float) * c * nb, st), "workspace");
  } else {
    NPPB_CUDA(mxw.alloc(mx_workspace_bytes(count, n), st), "workspace");
    NPPB_CUDA(y32.alloc(sizeof(float) * c * (size_t)mx_padded(n) * nrhs, st), "workspace");
  }
  NPPB_CUDA(b32.alloc(sizeof(float) * c * nb, st), "workspace");
  NPPB_CUDA(rsm.alloc(sizeof(double) * c * n, st), "workspace");
  NPPB_CUDA(csm.alloc(sizeof(double) * c * n, st), "workspace");
  NPPB_CUDA(cmx.alloc(sizeof(double) * c * n, st), "workspace");
  NPPB_CUDA(stm.alloc(sizeof(RefineState) * c, st), "workspace");
  NPPB_CUDA(cudaMemsetAsync(cmx.as<void>(), 0, sizeof(double) * c * n, st), "memset");
  NPPB_CUDA(cudaMemsetAsync(stm.as<void>(), 0, sizeof(RefineState) * c, st), "memset");
  NPPB_CUDA(info32.alloc(sizeof(int32_t) * c, st), "workspace");
  NPPB_CUDA(act.alloc(sizeof(int), st), "workspace");
  RefineState* S = stm.as<RefineState>();
  const bool equil = !(flags & NPPB_MIXED_NO_EQUILIBRATE);
  if (blocked) {
    NPPB_CUDA(mixed_equil_scan(dA, count, n, equil ? 1 : 0, rsm.as<double>(), cmx.as<double>(), S, st),
              "equilibrate");
  } else {
    NPPB_CUDA(mixed_equilibrate(dA, count, n, equil ? 1 : 0, a32.as<float>(), rsm.as<double>(), csm.as<double>(),
                                cmx.as<double>(), S, st),
              "equilibrate");
  }
  NPPB_CUDA(mixed_scale_rhs(dB, count, n, nrhs, rsm.as<double>(), b32.as<float>(), S, st), "scale rhs");

  std::vector<RefineState> hs(c);
  std::vector<int32_t> fallback(c, 0);
  bool any_fallback = false;
  if (blocked) {
    MxBufs mb;
    mx_carve(mb, mxw.as<void>(), count, n);
    NPPB_CUDA(mx_build(dA, rsm.as<double>(), cmx.as<double>(), equil ? 1 : 0, csm.as<double>(), S, mb, st),
              "butterfly transform");
    NPPB_CUDA(mx_factor(mb, st), "FP32 block factorisation");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    if (mx_timeouts_take() != 0) {
      set_error("tensor-core block factorisation: a completion wait ran out");
      return NPPB_E_CUDA;
    }
    NPPB_CUDA(mixed_mark_fp32_failures(mb.info, S, count, st), "mark");
    float* Y = y32.as<float>();
    NPPB_CUDA(mx_rhs_in(b32.as<float>(), Y, nrhs, S, 0, mb, st), "transform rhs");
    NPPB_CUDA(mx_solve(Y, nrhs, S, 0, mb, st), "FP32 solve");
    NPPB_CUDA(mx_apply(Y, dX, csm.as<double>(), nrhs, S, 1, mb, st), "apply");
    int h_act = 0;
    if (!gmres) {
      for (int it = 0;; ++it) {
        NPPB_CUDA(cudaMemsetAsync(act.as<int>(), 0, sizeof(int), st), "memset");
        // the scaled residual lands in b32 (row order of A)
        NPPB_CUDA(mixed_residual(dA, dB, dX, count, n, nrhs, rsm.as<double>(), b32.as<float>(), nullptr, S, tol,
                                 it, max_iter, 1, act.as<int>(), st),
                  "residual");
        NPPB_CUDA(cudaMemcpyAsync(&h_act, act.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st), "readback");
        NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
        if (h_act == 0 || it >= max_iter) break;
        NPPB_CUDA(mx_rhs_in(b32.as<float>(), Y, nrhs, S, 1, mb, st), "transform residual");
        NPPB_CUDA(mx_solve(Y, nrhs, S, 1, mb, st), "FP32 correction solve");
        NPPB_CUDA(mx_apply(Y, dX, csm.as<double>(), nrhs, S, 0, mb, st), "apply");
      }
    } else {
      // GMRES-IR: each correction by LU-preconditioned GMRES in FP64 (the
      // preconditioner is the FP32 factorisation applied to FP64 vectors)
      const size_t vec = c * nb;  // doubles of one vector plane (count x n x nrhs)
      DevMem gV, gR, gY, gW, gS, gA;
      NPPB_CUDA(gV.alloc(sizeof(double) * vec * (kGmM + 1), st), "workspace");
      NPPB_CUDA(gR.alloc(sizeof(double) * vec, st), "workspace");
      NPPB_CUDA(gY.alloc(sizeof(double) * c * (size_t)mb.N * nrhs, st), "workspace");
      NPPB_CUDA(gW.alloc(sizeof(double) * vec, st), "workspace");
      NPPB_CUDA(gS.alloc(sizeof(GmState) * c * nrhs, st), "workspace");
      NPPB_CUDA(gA.alloc(sizeof(int), st), "workspace");
      double* V = gV.as<double>();
      auto precond = [&](const double* in, double* out) -> int {  // out = M^-1 in (in: already row-scaled)
        NPPB_CUDA(mx_rhs_in64(in, gY.as<double>(), nrhs, S, 1, mb, st), "transform");
        NPPB_CUDA(mx_solve64(gY.as<double>(), nrhs, S, 1, mb, st), "preconditioner solve");
        NPPB_CUDA(mx_apply64(gY.as<double>(), out, csm.as<double>(), nrhs, S, 1, mb, st), "apply");
        return NPPB_OK;
      };
      for (int it = 0;; ++it) {
        NPPB_CUDA(cudaMemsetAsync(act.as<int>(), 0, sizeof(int), st), "memset");
        NPPB_CUDA(mixed_residual(dA, dB, dX, count, n, nrhs, rsm.as<double>(), nullptr, nullptr, S, tol, it,
                                 max_iter, 1, act.as<int>(), st, gR.as<double>()),
                  "residual");
        NPPB_CUDA(cudaMemcpyAsync(&h_act, act.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st), "readback");
        NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
        if (h_act == 0 || it >= max_iter) break;
        NPPB_RC(precond(gR.as<double>(), gW.as<double>()));
        NPPB_CUDA(gm_start(gW.as<double>(), V, gS.as<GmState>(), S, count, n, nrhs, st), "GMRES start");
        for (int k = 0; k < kGmM; ++k) {
          NPPB_CUDA(mixed_matvec(dA, V + (size_t)k * vec, count, n, nrhs, rsm.as<double>(), gR.as<double>(), S, st),
                    "GMRES product");
          NPPB_RC(precond(gR.as<double>(), gW.as<double>()));
          int h_in = 0;
          NPPB_CUDA(cudaMemsetAsync(gA.as<int>(), 0, sizeof(int), st), "memset");
          NPPB_CUDA(gm_arnoldi(gW.as<double>(), V, gS.as<GmState>(), S, count, n, nrhs, k, kGmresTau, gA.as<int>(),
                               st),
                    "GMRES step");
          NPPB_CUDA(cudaMemcpyAsync(&h_in, gA.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st), "readback");
          NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
          if (h_in == 0) break;
        }
        NPPB_CUDA(gm_update(V, dX, gS.as<GmState>(), S, count, n, nrhs, st), "GMRES update");
      }
    }
    NPPB_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(RefineState) * c, cudaMemcpyDeviceToHost, st), "readback");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    for (size_t s = 0; s < c; ++s) {
      if (hs[s].status != kRefineConverged && !(flags & NPPB_MIXED_NO_FALLBACK)) {
        fallback[s] = 1;
        any_fallback = true;
      }
    }
  } else if (n > 32) {
    StepArgsT<float> sa{};
    sa.scratch = sc32.as<StepScratchT<float>>();
    sa.A = nullptr;  // factor the scaled FP32 matrix in place
    sa.LU = a32.as<float>();
    sa.ipiv = piv.as<int32_t>();
    sa.B = b32.as<float>();
    sa.X = y32.as<float>();
    sa.info = info32.as<int32_t>();
    sa.un = n;
    sa.unrhs = nrhs;
    sa.uleft = 1;
    const bool tc = (flags & NPPB_MIXED_TCGEN05) != 0;
    sa.umode = (flags & NPPB_MIXED_BF16) ? 2
               : (flags & NPPB_MIXED_TF32) ? (tc ? 4 : 1)
               : (flags & NPPB_MIXED_FP32_FMA) ? 0
               : (tc ? 5 : 3);
    NPPB_CUDA(run_step_uniform<float>(sa, count, st), "FP32 factorisation");
    if (tc && (sa.umode == 4 || sa.umode == 5)) {
      NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
      if (tc_timeouts_take() != 0) {
        set_error("tensor-core trailing update: a completion wait ran out");
        return NPPB_E_CUDA;
      }
    }
    NPPB_CUDA(mixed_mark_fp32_failures(info32.as<int32_t>(), S, count, st), "mark");
    NPPB_CUDA(mixed_row_positions(piv.as<int32_t>(), count, n, rpos.as<int32_t>(), st), "row positions");
    NPPB_CUDA(mixed_apply(dX, y32.as<float>(), csm.as<double>(), count, n, nrhs, S, 1, st), "apply");
    int h_act = 0;
    for (int it = 0;; ++it) {
      NPPB_CUDA(cudaMemsetAsync(act.as<int>(), 0, sizeof(int), st), "memset");
      // the scaled residual lands in y32 already in pivoted row order
      NPPB_CUDA(mixed_residual(dA, dB, dX, count, n, nrhs, rsm.as<double>(), y32.as<float>(), rpos.as<int32_t>(), S,
                               tol, it, max_iter, 1, act.as<int>(), st),
                "residual");
      NPPB_CUDA(cudaMemcpyAsync(&h_act, act.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, st), "readback");
      NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
      if (h_act == 0 || it >= max_iter) break;
      StepArgsT<float> sb = sa;  // correction: solve with the stored FP32 factors, in place on y32
      sb.B = nullptr;
      sb.X = y32.as<float>();
      NPPB_CUDA(run_step_solve_uniform<float>(sb, count, st, true), "FP32 correction solve");
      NPPB_CUDA(mixed_apply(dX, y32.as<float>(), csm.as<double>(), count, n, nrhs, S, 0, st), "apply");
    }
    NPPB_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(RefineState) * c, cudaMemcpyDeviceToHost, st), "readback");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    for (size_t s = 0; s < c; ++s) {
      if (hs[s].status != kRefineConverged && !(flags & NPPB_MIXED_NO_FALLBACK)) {
        fallback[s] = 1;
        any_fallback = true;
      }
    }
  } else {
    // orders <= 32 are one warp-resident FP64 solve already: no refinement to gain
    std::fill(fallback.begin(), fallback.end(), 1);
    any_fallback = true;
  }

  std::vector<int32_t> hinfo(c, 0);
  if (any_fallback) {
    std::vector<int> idx;
    for (size_t s = 0; s < c; ++s)
      if (fallback[s]) idx.push_back((int)s);
    const size_t k = idx.size();
    DevMem ca, cb, cx, ci;
    NPPB_CUDA(ca.alloc(sizeof(double) * k * nn, st), "fallback workspace");
    NPPB_CUDA(cb.alloc(sizeof(double) * k * nb, st), "fallback workspace");
    NPPB_CUDA(cx.alloc(sizeof(double) * k * nb, st), "fallback workspace");
    NPPB_CUDA(ci.alloc(sizeof(int32_t) * k, st), "fallback workspace");
    for (size_t q = 0; q < k; ++q) {
      const size_t s = idx[q];
      NPPB_CUDA(cudaMemcpyAsync(ca.as<double>() + q * nn, dA + s * nn, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st),
                "gather");
      NPPB_CUDA(cudaMemcpyAsync(cb.as<double>() + q * nb, dB + s * nb, sizeof(double) * nb, cudaMemcpyDeviceToDevice, st),
                "gather");
    }
    NPPB_RC(nppb_d_linalg_batched((int64_t)k, n, nrhs, NPPB_WANT_SOLVE, ca.as<double>(), cb.as<double>(),
                                  cx.as<double>(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                  ci.as<int32_t>(), st));
    for (size_t q = 0; q < k; ++q) {
      const size_t s = idx[q];
      NPPB_CUDA(cudaMemcpyAsync(dX + s * nb, cx.as<double>() + q * nb, sizeof(double) * nb, cudaMemcpyDeviceToDevice, st),
                "scatter");
    }
    std::vector<int32_t> cinfo(k);
    if (k) NPPB_CUDA(cudaMemcpyAsync(cinfo.data(), ci.as<int32_t>(), sizeof(int32_t) * k, cudaMemcpyDeviceToHost, st),
                     "readback");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    for (size_t q = 0; q < k; ++q) hinfo[idx[q]] = cinfo[q];
  }
  // final backward error of every system, whatever path produced it (the last
  // residual of the refinement already is, unless some system fell back)
  if (any_fallback || n <= 32)
    NPPB_CUDA(mixed_residual(dA, dB, dX, count, n, nrhs, rsm.as<double>(), nullptr, nullptr, S, tol, 0, max_iter,
                             0, act.as<int>(), st),
              "residual");
  if (dFerr && dXtrue) NPPB_CUDA(mixed_ferr(dX, dXtrue, count, n, nrhs, dFerr, st), "forward error");
  NPPB_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(RefineState) * c, cudaMemcpyDeviceToHost, st), "readback");
  NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
  std::vector<double> berr(c);
  std::vector<int32_t> iters(c);
  for (size_t s = 0; s < c; ++s) {
    berr[s] = hs[s].eta;
    iters[s] = n > 32 ? hs[s].iters : 0;
  }
  if (dBerr) NPPB_CUDA(cudaMemcpyAsync(dBerr, berr.data(), sizeof(double) * c, cudaMemcpyHostToDevice, st), "write");
  if (dIters) NPPB_CUDA(cudaMemcpyAsync(dIters, iters.data(), sizeof(int32_t) * c, cudaMemcpyHostToDevice, st), "write");
  if (dFallback)
    NPPB_CUDA(cudaMemcpyAsync(dFallback, fallback.data(), sizeof(int32_t) * c, cudaMemcpyHostToDevice, st), "write");
  if (dinfo) NPPB_CUDA(cudaMemcpyAsync(dinfo, hinfo.data(), sizeof(int32_t) * c, cudaMemcpyHostToDevice, st), "write");
  NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
  return NPPB_OK;
}

template <class F>
int guarded(F&& f) {
  try {
    clear_error();
    return f();
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return NPPB_E_NOMEM;
  }
}

}  // namespace

extern "C" {

int nppb_d_solve_mixed_batched(int64_t count, int32_t n, int32_t nrhs, const double* dA, const double* dB,
                               double* dX, const double* dXtrue, double tol, int32_t max_iter, int flags,
                               int32_t* dinfo, double* dBerr, double* dFerr, int32_t* dIters,
                               int32_t* dFallback, void* stream) {
  return guarded([&]() -> int {
    return mixed(count, n, nrhs, dA, dB, dX, dXtrue, tol, max_iter, flags, dinfo, dBerr, dFerr, dIters,
                 dFallback, static_cast<cudaStream_t>(stream));
  });
}

int nppb_solve_mixed_batched(int64_t count, int32_t n, int32_t nrhs, const double* A, const double* B, double* X,
                             const double* Xtrue, double tol, int32_t max_iter, int flags, int32_t* info,
                             double* berr, double* ferr, int32_t* iters, int32_t* fallback) {
  return guarded([&]() -> int {
    if (count <= 0 || n <= 0 || nrhs <= 0) {
      if (count < 0 || n < 0 || nrhs < 0) {
        set_error("negative count, order or nrhs");
        return NPPB_E_ARG;
      }
      return NPPB_OK;
    }
    if (!device()) return NPPB_E_NODEV;
    cudaStream_t st = thread_stream();
    const size_t nn = (size_t)count * n * n, nb = (size_t)count * n * nrhs, c = (size_t)count;
    DevMem dA, dB, dX, dT, dI, dBe, dFe, dIt, dFb;
    NPPB_CUDA(dA.alloc(sizeof(double) * nn, st), "allocation");
    NPPB_CUDA(dB.alloc(sizeof(double) * nb, st), "allocation");
    NPPB_CUDA(dX.alloc(sizeof(double) * nb, st), "allocation");
    NPPB_CUDA(dI.alloc(sizeof(int32_t) * c, st), "allocation");
    NPPB_CUDA(dBe.alloc(sizeof(double) * c, st), "allocation");
    NPPB_CUDA(dFe.alloc(sizeof(double) * c, st), "allocation");
    NPPB_CUDA(dIt.alloc(sizeof(int32_t) * c, st), "allocation");
    NPPB_CUDA(dFb.alloc(sizeof(int32_t) * c, st), "allocation");
    if (Xtrue) NPPB_CUDA(dT.alloc(sizeof(double) * nb, st), "allocation");
    NPPB_CUDA(cudaMemcpyAsync(dA.as<double>(), A, sizeof(double) * nn, cudaMemcpyHostToDevice, st), "copy");
    NPPB_CUDA(cudaMemcpyAsync(dB.as<double>(), B, sizeof(double) * nb, cudaMemcpyHostToDevice, st), "copy");
    if (Xtrue) NPPB_CUDA(cudaMemcpyAsync(dT.as<double>(), Xtrue, sizeof(double) * nb, cudaMemcpyHostToDevice, st), "copy");
    NPPB_RC(mixed(count, n, nrhs, dA.as<double>(), dB.as<double>(), dX.as<double>(), Xtrue ? dT.as<double>() : nullptr,
                  tol, max_iter, flags, dI.as<int32_t>(), dBe.as<double>(), dFe.as<double>(), dIt.as<int32_t>(),
                  dFb.as<int32_t>(), st));
    NPPB_CUDA(cudaMemcpyAsync(X, dX.as<double>(), sizeof(double) * nb, cudaMemcpyDeviceToHost, st), "copy");
    if (info) NPPB_CUDA(cudaMemcpyAsync(info, dI.as<int32_t>(), sizeof(int32_t) * c, cudaMemcpyDeviceToHost, st), "copy");
    if (berr) NPPB_CUDA(cudaMemcpyAsync(berr, dBe.as<double>(), sizeof(double) * c, cudaMemcpyDeviceToHost, st), "copy");
    if (ferr && Xtrue)
      NPPB_CUDA(cudaMemcpyAsync(ferr, dFe.as<double>(), sizeof(double) * c, cudaMemcpyDeviceToHost, st), "copy");
    if (iters) NPPB_CUDA(cudaMemcpyAsync(iters, dIt.as<int32_t>(), sizeof(int32_t) * c, cudaMemcpyDeviceToHost, st), "copy");
    if (fallback)
      NPPB_CUDA(cudaMemcpyAsync(fallback, dFb.as<int32_t>(), sizeof(int32_t) * c, cudaMemcpyDeviceToHost, st), "copy");
    NPPB_CUDA(cudaStreamSynchronize(st), "synchronize");
    return NPPB_OK;
  });
}

}  // extern "C"
