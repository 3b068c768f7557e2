/*
 * numpp_b200.h — C ABI of the B200-native (sm_100a) batched dense linear-solve
 * path for NumPP: numpp::linalg::solve / inv / det / slogdet on stacked
 * (..., n, n) float64 arrays, and the matmul they rest on.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and is
 * thread-safe. Arrays are C-contiguous (row-major). Host-buffer entry points
 * copy in, compute on the GPU and copy out before returning, exactly like a
 * NumPP GpuVTable slot (the caller owns every buffer; nothing is retained).
 * Device-buffer entry points (prefix nppb_d_) take device pointers and a CUDA
 * stream (cudaStream_t passed as void*; NULL = the legacy default stream) and
 * only enqueue work.
 *
 * Status codes: NPPB_OK (0) on success; NPPB_DECLINED (1) when the request is
 * outside what the GPU path serves (dtype, op), so a NumPP dispatcher falls
 * back to its portable CPU kernel; negative values are errors, described by
 * nppb_last_error() on the calling thread. A singular matrix is not an error:
 * the per-system info[] entry is set to k+1 for the first exactly-zero pivot
 * k (0-based), mirroring where the reference stops.
 *
 * Pivots (ipiv) are LAPACK-style swap lists, 0-based: at step k rows k and
 * ipiv[k] were exchanged. The reference's permutation vector piv
 * (src/linalg/linalg.cpp:52,60 in NumPP) is the identity with those swaps
 * applied in order.
 */
#ifndef NUMPP_B200_H
#define NUMPP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NPPB_ABI_VERSION 1

enum {
  NPPB_OK = 0,
  NPPB_DECLINED = 1,
  NPPB_E_ARG = -1,      /* invalid argument (shape, null pointer, size)      */
  NPPB_E_NODEV = -2,    /* no usable sm_100 device                           */
  NPPB_E_CUDA = -3,     /* a CUDA runtime call failed                        */
  NPPB_E_NOMEM = -4,    /* device allocation failed or budget exceeded      */
  NPPB_E_RANGE = -5     /* size outside what this entry point supports      */
};

/* numpp::DTypeId values (include/numpp/core/dtype.hpp:16-22 in NumPP). */
enum { NPPB_DT_FLOAT32 = 10, NPPB_DT_FLOAT64 = 11 };

/* ---- library ---------------------------------------------------------- */
int nppb_abi_version(void);
/* 1 when a compute-capability 10.x device is present (numpp gpu_vtable() is
 * non-null exactly then: src/backend/cuda_backend.cu:120-123,320). */
int nppb_device_available(void);
/* Message for the last failing call on this thread ("" if none). */
const char* nppb_last_error(void);
/* Largest order served by the batched entry points. */
int32_t nppb_max_order(void);
/* The numpp::GpuVTable this library provides (numpp::gpu_vtable(), see
 * include/numpp/backend/gpu_vtable.hpp), for hosts that cannot name the C++
 * symbol; NULL when no compute-capability 10.x device is present. */
const void* nppb_gpu_vtable(void);

/* ---- GpuVTable slots (include/numpp/backend/gpu_vtable.hpp:17-26) ------ */
/* The elementwise/reduce slots are called by NumPP's ufunc layer without a
 * null check (src/umath/ufunc.cpp:528-531,539-541,611-613); this backend
 * declines them (returns NPPB_DECLINED) so the portable kernels run. */
int nppb_elementwise_binary(int op, int dtype, int64_t n, const void* a, const void* b, void* out);
int nppb_elementwise_unary(int op, int dtype, int64_t n, const void* a, void* out);
int nppb_reduce(int op, int dtype, int64_t n, const void* a, void* out);
/* GpuVTable::gemm (gpu_vtable.hpp:22-26; the CUDA backend's gemm_impl at
 * src/backend/cuda_backend.cu:288-293): row-major C[m,n] = A[m,k] B[k,n],
 * float32 or float64, host buffers. */
int nppb_gemm(int dtype, int64_t m, int64_t n, int64_t k, const void* A, const void* B, void* C);
/* Same on device buffers (FP64 runs on DMMA). */
int nppb_d_gemm(int dtype, int64_t m, int64_t n, int64_t k, const void* dA, const void* dB,
                void* dC, void* stream);

/* Stacked matmul: `batch` contiguous row-major FP64 products C[z] = A[z] B[z]
 * (m x k times k x n) on the DMMA GEMM, one launch for the whole stack. The
 * reference's matmul is 2-D only (src/backend/backend.cpp:121-177 rejects
 * ndim > 2); this is the einsum 'bij,bjk->bik' its callers fall back to. */
int nppb_d_gemm_batched(int64_t batch, int64_t m, int64_t n, int64_t k, const double* dA, const double* dB,
                        double* dC, void* stream);
int nppb_gemm_batched(int64_t batch, int64_t m, int64_t n, int64_t k, const double* A, const double* B,
                      double* C);
/* matrix_power over a (count, n, n) FP64 stack (src/linalg/batched.cpp:83-84
 * mapping src/linalg/linalg.cpp:440-454): binary exponentiation with the
 * batched GEMM, the batched inverse first when p < 0 (info[i] != 0: system i
 * is singular, its R is then undefined), the identity for p = 0. */
int nppb_matrix_power_batched(int64_t count, int32_t n, int64_t p, const double* A, double* R, int32_t* info);
/* cholesky over a (count, n, n) FP64 stack (src/linalg/linalg.cpp:117-136;
 * stacks src/linalg/batched.cpp:77): lower-triangular L with A = L L^T, read
 * from A's lower triangle only. info[i] = k > 0: system i is not positive
 * definite (its k-th pivot is <= 0; the reference raises "Matrix is not
 * positive definite"); L of that system is then undefined. Orders <= 4096. */
int nppb_cholesky_batched(int64_t count, int32_t n, const double* A, double* L, int32_t* info);
/* lstsq over `count` problems of one shape (src/linalg/linalg.cpp:755-784;
 * its SVD :620-712): A (count, m, n), B (count, m, k) row-major; per problem
 * X (n, k) = pinv(A) B with singular values below
 * tol = (rcond < 0 ? eps * max(m, n) : rcond) * s_max dropped, S
 * (min(m, n), descending), rank, and resid (k) with has_resid = 1 when
 * m > n and rank == n (else resid is not written, as the reference returns
 * no residuals). k = 0: singular values and rank only (B, X, resid, has_resid
 * may be NULL). NPPB_DECLINED past min(m, n) = 64, k = 64 or about
 * m * n + min(m, n)^2 = 26000 (one problem's matrices must fit in shared
 * memory): the CPU path keeps those. */
int nppb_lstsq_batched(int64_t count, int32_t m, int32_t n, int32_t k, const double* A, const double* B,
                       double rcond, double* X, double* S, int32_t* rank, double* resid, int32_t* has_resid);
int nppb_d_lstsq_batched(int64_t count, int32_t m, int32_t n, int32_t k, const double* dA, const double* dB,
                         double rcond, double* dX, double* dS, int32_t* drank, double* dres, int32_t* dhas,
                         void* stream);
/* The same on device buffers, enqueued on `stream` (workspace allocated
 * stream-ordered for the call). */
int nppb_d_cholesky_batched(int64_t count, int32_t n, const double* dA, double* dL, int32_t* dinfo,
                            void* stream);

/* ---- uniform batches: count systems of order n (host buffers) ----------- */
/* getrf: LU with partial pivoting in place (src/linalg/linalg.cpp:48-71),
 * A (count,n,n) overwritten by the unit-lower L and U in pivoted row order. */
int nppb_getrf_batched(int64_t count, int32_t n, double* A, int32_t* ipiv, int32_t* info);
/* getrs: B (count,n,nrhs) overwritten by the solution (linalg.cpp:73-90). */
int nppb_getrs_batched(int64_t count, int32_t n, int32_t nrhs, const double* LU,
                       const int32_t* ipiv, double* B);
/* numpp::linalg::solve on a (count,n,n) stack with a (count,n,nrhs) right-hand
 * side (linalg.cpp:368-385, src/linalg/batched.cpp:90-100). */
int nppb_solve_batched(int64_t count, int32_t n, int32_t nrhs, const double* A, const double* B,
                       double* X, int32_t* info);
/* numpp::linalg::inv (linalg.cpp:386-392, 105-115; batched.cpp:75). */
int nppb_inv_batched(int64_t count, int32_t n, const double* A, double* Ainv, int32_t* info);
/* numpp::linalg::det (linalg.cpp:393-407; batched.cpp:76). Singular -> 0. */
int nppb_det_batched(int64_t count, int32_t n, const double* A, double* det);
/* numpp::linalg::slogdet (linalg.cpp:408-439; batched.cpp:102-108).
 * Singular -> sign 0, logabsdet -inf. */
int nppb_slogdet_batched(int64_t count, int32_t n, const double* A, double* sign,
                         double* logabsdet);
/* solve and det from one factorisation (the reference factors twice). */
int nppb_solve_det_batched(int64_t count, int32_t n, int32_t nrhs, const double* A,
                           const double* B, double* X, double* det, int32_t* info);

/* ---- uniform batches on device buffers --------------------------------- */
/* `flags` selects outputs: NPPB_WANT_* below. Null output pointers are
 * allowed for outputs not selected. dLU/dipiv are the factor workspace
 * (count*n*n doubles, count*n int32); pass NULL to let the library allocate
 * it stream-ordered for the call. With NPPB_WANT_LU the factors stay there. */
enum {
  NPPB_WANT_LU = 1,
  NPPB_WANT_SOLVE = 2,
  NPPB_WANT_DET = 4,
  NPPB_WANT_SLOGDET = 8,
  NPPB_WANT_INV = 16
};
int nppb_d_linalg_batched(int64_t count, int32_t n, int32_t nrhs, int flags, const double* dA,
                          const double* dB, double* dX, double* dInv, double* dDet,
                          double* dSign, double* dLogabs, double* dLU, int32_t* dipiv,
                          int32_t* dinfo, void* stream);
/* getrs from factors left by nppb_d_linalg_batched(NPPB_WANT_LU): dB -> dX
 * (dX may equal dB). */
int nppb_d_getrs_batched(int64_t count, int32_t n, int32_t nrhs, const double* dLU,
                         const int32_t* dipiv, const double* dB, double* dX, void* stream);

/* Allocation-free solve. No counterpart in the reference: NumPP's CUDA
 * backend allocates per call (src/backend/cuda_backend.cu:126-146,189-206).
 * For callers that must not allocate device memory while they run (hosts
 * whose device memory is reserved up front, fixed-pool allocators where a
 * cudaMalloc would fail or stall): X = A^-1 B for a uniform batch on device
 * buffers, with no cudaMalloc / cudaFree or allocating call. Orders above 32
 * use a fixed 32 MiB scratch array inside the library, so
 * count * (8*n*n + 8616) bytes must fit in 32 MiB (NPPB_E_RANGE otherwise,
 * before any GPU work); orders up to 32 need no scratch. The array belongs to
 * the library's module: its 32 MiB are reserved on every device where the
 * module is loaded (each context under eager module loading, the first use
 * under lazy loading) until the process exits. The first call on each device
 * looks up the array's device address, so make that first call before any
 * stream capture. Every call shares the array: calls that overlap on the GPU
 * (other streams, other threads) race and must be ordered by the caller.
 * Always the single-level step schedule (NPPB_BLOCKED_MIN_N is ignored).
 * info as for the other solves; dX must not alias dB. */
int nppb_d_solve_batched_noalloc(int64_t count, int32_t n, int32_t nrhs, const double* dA,
                                 const double* dB, double* dX, int32_t* dinfo, void* stream);

/* ---- mixed precision: FP32 factors, FP64 iterative refinement ---------- */
/* No counterpart in the reference (NumPP solves in double only,
 * src/linalg/linalg.cpp:92-103). X = A^-1 B for a uniform batch: power-of-two
 * row/column equilibration, an LU in FP32, then FP64 refinement (R = B - A X
 * in FP64, correction solved with the FP32 factors, added in FP64) until the
 * normwise backward error eta = max|R| / (||A||_inf max|X| + max|B|) <= tol.
 * A system is stalled when its eta stops decreasing, or when the contraction
 * it has shown cannot bring eta to tol within the corrections left; stalled
 * systems, FP32 zero pivots and systems still refining after max_iter
 * corrections are refactored and solved in FP64. Per system: berr (final eta), ferr
 * (max|X - Xtrue| / max|Xtrue|, when Xtrue is given), iters (corrections
 * applied), fallback (1 = the FP64 solve ran), info (of the FP64 solve, when
 * it ran). Orders <= 32 always take the FP64 warp kernel (fallback = 1). The
 * device form synchronises `stream` (it reads convergence counts back between
 * corrections).
 * The FP32 factorisation, by default: the equilibrated matrix mixed by a
 * depth-2 random butterfly transform on both sides, padded to a multiple of
 * 128 with an identity block, and factored in 128-column blocks with partial
 * pivoting among each diagonal block's own rows; each block's two triangular
 * solves (by the inverses of its diagonal factors) and its trailing update
 * run as tcgen05 GEMMs with error-compensated TF32 products (each operand
 * split into two TF32 parts, three products: close to FP32 accuracy) and TMEM
 * accumulators, operands staged by TMA. The refinement works on the original
 * matrix: the transform and the restricted pivoting change which factors
 * precondition the corrections, not the system solved.
 * With NPPB_MIXED_PIVOTED (or any of TF32 / BF16 / FP32_FMA / TCGEN05): LU
 * with partial pivoting on the step-wise kernels; trailing products as
 * error-compensated TF32 (default), one TF32 or BF16 product (NPPB_MIXED_TF32
 * / NPPB_MIXED_BF16), or FP32 fused multiply-adds (NPPB_MIXED_FP32_FMA); the
 * TF32 products on mma.sync, or with NPPB_MIXED_TCGEN05 on tcgen05 with TMEM
 * accumulators. FP32 accumulation in every case; the stored factors and the
 * correction solves stay FP32.
 * With NPPB_MIXED_GMRES (default factorisation only): each correction is
 * solved by GMRES on M^-1 A d = M^-1 R (Carson and Higham's GMRES-based
 * refinement), M^-1 the FP32 factorisation applied to FP64 vectors with FP64
 * accumulation, FP64 Krylov vectors and products with A, up to 30 Arnoldi
 * steps per correction (to a relative residual of 1e-6); it reaches tol for
 * conditioning the plain refinement stalls on (kappa up to about 1e8 with
 * FP32 factors). iters then counts outer corrections. */
enum {
  NPPB_MIXED_NO_EQUILIBRATE = 1,
  NPPB_MIXED_NO_FALLBACK = 2,
  NPPB_MIXED_TF32 = 4,
  NPPB_MIXED_BF16 = 8,
  NPPB_MIXED_FP32_FMA = 16,
  NPPB_MIXED_TCGEN05 = 32,
  NPPB_MIXED_PIVOTED = 64,
  NPPB_MIXED_GMRES = 128
};
int nppb_d_solve_mixed_batched(int64_t count, int32_t n, int32_t nrhs, const double* dA,
                               const double* dB, double* dX, const double* dXtrue, double tol,
                               int32_t max_iter, int flags, int32_t* dinfo, double* dBerr,
                               double* dFerr, int32_t* dIters, int32_t* dFallback, void* stream);
int nppb_solve_mixed_batched(int64_t count, int32_t n, int32_t nrhs, const double* A, const double* B,
                             double* X, const double* Xtrue, double tol, int32_t max_iter, int flags,
                             int32_t* info, double* berr, double* ferr, int32_t* iters,
                             int32_t* fallback);

/* ---- serving loop ---------------------------------------------------------- */
/* No counterpart in the reference (NumPP solves one call at a time on the
 * caller's thread, src/linalg/linalg.cpp:368-385). A server owns one worker
 * thread, one stream and a resident-factor arena carved out of budget_bytes
 * of device memory (three quarters; the rest bounds each batch's inputs).
 * Requests from any thread are batched continuously: a batch closes when its
 * oldest request has waited window_us, or at max_batch requests. A request
 * either factors A (n x n, row-major) and solves for B (n x nrhs) into X,
 * optionally keeping the factors resident (*factor_out = their id), or
 * re-solves new right-hand sides with a resident factor (A == NULL,
 * factor_in = its id). A, B and X are read / written by the worker with
 * cudaMemcpyAsync and must stay valid until nppb_server_wait returns for the
 * request (pinned host memory takes the fast path). When a new factor does
 * not fit, the least recently used resident factors not read by the current
 * batch are evicted; a re-solve on an evicted factor completes with
 * NPPB_E_RANGE. A singular factorisation completes with NPPB_OK and
 * info = first zero pivot + 1 (the factor is then not kept). A request's
 * result does not depend on which other requests share its batch. */
typedef struct nppb_server nppb_server;
int nppb_server_create(nppb_server** srv, int64_t budget_bytes, double window_us, int32_t max_batch);
int nppb_server_submit(nppb_server* srv, int32_t n, int32_t nrhs, const double* A, const double* B, double* X,
                       int64_t factor_in, int32_t keep_factor, int64_t* request_id, int64_t* factor_out);
/* Waits up to timeout_s; NPPB_DECLINED if the request is still running then
 * (wait again). Otherwise returns the request's status, once per request,
 * with its info and its latency (submission to completion, seconds). */
int nppb_server_wait(nppb_server* srv, int64_t request_id, double timeout_s, int32_t* info,
                     double* latency_s);
int nppb_server_release_factor(nppb_server* srv, int64_t factor_id);
/* out6: requests completed, batches run, resident factors, arena bytes in
 * use, evictions, requests queued. */
int nppb_server_stats(nppb_server* srv, int64_t* out6);
/* Drains the queue, stops the worker, frees the arena. */
int nppb_server_destroy(nppb_server* srv);

/* ---- uneven batches ------------------------------------------------------ */
/* A plan packs `count` systems of different orders n[i] and right-hand-side
 * counts nrhs[i] into size classes (one warp-kernel launch per class of
 * orders <= 32; one chain of panel / row-move / update / substitution
 * launches per class above, chains on parallel graph branches) and replays
 * them as one CUDA graph. System i's matrix starts at element
 * a_off[i] of the packed A array, its right-hand side / solution at b_off[i]
 * of B / X, and its inverse (when inv_off[i] >= 0) at inv_off[i] of Inv.
 * Per-system outputs (sign, logabsdet, det, info) are indexed by i.
 * `flags` is a NPPB_WANT_* mask (NPPB_WANT_LU is ignored). */
typedef struct nppb_plan nppb_plan;
int nppb_plan_create(nppb_plan** plan, int64_t count, const int32_t* n, const int32_t* nrhs,
                     const int64_t* a_off, const int64_t* b_off, const int64_t* inv_off,
                     int flags);
/* Sizes (elements) the packed arrays must have. */
int nppb_plan_sizes(const nppb_plan* plan, int64_t* a_elems, int64_t* b_elems,
                    int64_t* inv_elems);
/* Device buffers; enqueues on `stream`. */
int nppb_plan_execute(nppb_plan* plan, const double* dA, const double* dB, double* dX,
                      double* dInv, double* dDet, double* dSign, double* dLogabs,
                      int32_t* dinfo, void* stream);
/* Autotuner (no reference counterpart): times the plan with 1, 2, 3, 4 and 6
 * independent step chains (graph branches whose panels overlap each other's
 * updates), each with and without look-ahead (the next panels overlapping
 * the current trailing update inside a chain), on these device buffers, a
 * warm-up and two replays each, and keeps the fastest; *chains_out = the
 * chain count kept, negated when look-ahead is on; *ms_out = its time per
 * execution. The outputs are written as by nppb_plan_execute; synchronises
 * `stream`. */
int nppb_plan_autotune(nppb_plan* plan, const double* dA, const double* dB, double* dX, double* dInv,
                       double* dDet, double* dSign, double* dLogabs, int32_t* dinfo, void* stream,
                       int32_t* chains_out, float* ms_out);
/* The autotuner's on-disk cache: nppb_plan_autotune first looks its key up
 * (and on a hit builds the cached configuration and runs it once, untimed,
 * *ms_out = the cached time), otherwise tunes and appends the result. The
 * file is $NPPB_AUTOTUNE_CACHE (an empty value disables the cache), else
 * $XDG_CACHE_HOME/numpp_b200/autotune.txt, else ~/.cache/numpp_b200/autotune.txt;
 * one line per entry, "<key>\t<chains>\t<ms>" (chains negated with
 * look-ahead), the last line of a key winning. NPPB_AUTOTUNE_REFRESH=1 tunes
 * afresh. The key names the device (name, compute capability, SM count; "nodev"
 * without one), the flags and the batch's histogram over order class
 * (8, 16, 32, 64, ..., 4096) x right-hand-side class (0, 1, 8, 32, 64, more),
 * each count bucketed to its power of two. No device work in these three. */
int nppb_autotune_key(int64_t count, const int32_t* n, const int32_t* nrhs, int flags, char* buf, int64_t len);
int nppb_autotune_cache_get(const char* key, int32_t* chains, float* ms, int32_t* found);
int nppb_autotune_cache_put(const char* key, int32_t chains, float ms);
/* Host buffers: copies in, runs, copies out, synchronises. Inputs in pinned
 * memory take the fast DMA path. */
int nppb_plan_execute_host(nppb_plan* plan, const double* A, const double* B, double* X,
                           double* Inv, double* Det, double* Sign, double* Logabs,
                           int32_t* info);
int nppb_plan_destroy(nppb_plan* plan);
/* Introspection for measurement: the plan's size classes, each with its kernel
 * (1 = warp-per-system, 0 = CTA-per-system), order bound, system count and the
 * algorithmic flops / minimum bytes of what it computes (LAPACK counts:
 * getrf 2/3n^3-1/2n^2+5/6n, getrs 2n^2k-nk, inverse +4/3n^3). */
int nppb_plan_num_classes(const nppb_plan* plan);
/* Kernel launches one execution makes (graph nodes). */
int nppb_plan_num_launches(const nppb_plan* plan);
int nppb_plan_class_info(const nppb_plan* plan, int cls, int* is_warp, int* bound,
                         int64_t* systems, double* flops, double* bytes);
/* Runs every class alone on `stream`, `reps` launches each between two CUDA
 * events on that stream; ms_out[cls] = mean milliseconds of one launch. */
int nppb_plan_time_classes(nppb_plan* plan, const double* dA, const double* dB, double* dX,
                           double* dInv, double* dDet, double* dSign, double* dLogabs,
                           int32_t* dinfo, void* stream, int reps, float* ms_out);
/* Every launch of one execution, one after another on `stream`, each between
 * two CUDA events: ms_out[k] = summed milliseconds and flops_out[k] = the
 * arithmetic done, per kernel kind k: 0 warp-per-system LU (orders <= 32),
 * 1 panel factorisation, 2 strip update (row moves, U12, trailing update on
 * DMMA), 3 back substitution (and, for getrs plans, forward substitution). */
int nppb_plan_time_kernels(nppb_plan* plan, const double* dA, const double* dB, double* dX,
                           double* dInv, double* dDet, double* dSign, double* dLogabs,
                           int32_t* dinfo, void* stream, double* ms_out, double* flops_out);

/* One-shot uneven batch on host buffers (plan + execute + destroy). */
int nppb_solve_grouped(int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
                       const int64_t* b_off, const int64_t* inv_off, int flags, const double* A,
                       const double* B, double* X, double* Inv, double* Det, double* Sign,
                       double* Logabs, int32_t* info);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* NUMPP_B200_H */
