// Batched execution plan (host side). C++20.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include "nppb_internal.hpp"
#include "nppb_step.hpp"
#include "runtime.hpp"

namespace nppb {

class Plan {
 public:
  // Device pointers of one execution (A may be null: factor LU in place).
  struct Ptrs {
    const double* A;
    const double* B;
    double* X;
    double* Inv;
    double* Det;
    double* Sign;
    double* Logabs;
    int32_t* info;
    double* LU;
    int32_t* ipiv;
  };
  struct WarpClass {
    int bound;
    int64_t first, num;
    double flops, bytes;
  };
  struct PanelRange {
    int64_t first, num;
    int mmax;
  };
  struct Step {
    int k0 = 0;
    std::vector<PanelRange> panels;
    int64_t item_first = 0, item_count = 0;
    int64_t nfirst = 0;  // the first nfirst items: each system's first matrix strip (look-ahead)
    int nmax = 0;
  };
  // An independent sequence of steps over a subset of the step-wise systems;
  // chains run on separate graph branches so one chain's latency-bound panels
  // overlap another chain's tensor-core updates.
  struct Chain {
    std::vector<Step> steps;
    int64_t back_first = 0, back_count = 0;
    int nmax = 0;
    int64_t narrow_count = 0;  // the first narrow_count substitution strips: <= 8 columns, order > 512
    int narrow_nmax = 0;       // largest order among them
  };

  Plan() = default;
  Plan(const Plan&) = delete;
  Plan& operator=(const Plan&) = delete;
  ~Plan();

  // own_lu: allocate an LU workspace (else the factors go where A is: in place).
  // solve_only: getrs from factors already in LU / ipiv.
  // lu_off_ext / piv_off_ext: caller-placed factors (system i's LU at
  // lu_off_ext[i] of Ptrs::LU, its pivots at piv_off_ext[i] of Ptrs::ipiv).
  // Set alloc_stream before build for stream-ordered device allocations.
  int build(int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
            const int64_t* b_off, const int64_t* inv_off, int flags, bool solve_only, bool own_lu,
            const int64_t* lu_off_ext = nullptr, const int64_t* piv_off_ext = nullptr);
  int execute(const Ptrs& p, cudaStream_t st);
  cudaError_t launch_warp(const Ptrs& p, int cls, cudaStream_t st) const;
  cudaError_t launch_chain(const Ptrs& p, int chain, cudaStream_t st) const;
  // Every launch of one execution in order, each between two CUDA events on
  // `st`; ms[kind] accumulates the durations per kernel kind (KernelKind).
  int time_kernels(const Ptrs& p, cudaStream_t st, double* ms) const;
  cudaError_t launch_steps(const Ptrs& p, cudaStream_t st) const;  // every chain, in order
  int num_kernel_groups() const;
  // Work each kernel kind does per execution (flops of the arithmetic it runs,
  // triangular parts counted as triangles) and the launches per kind.
  enum KernelKind { kKindWarp = 0, kKindPanel = 1, kKindUpdate = 2, kKindBack = 3, kKinds = 4 };
  double kind_flops[kKinds] = {0, 0, 0, 0};
  int launches_per_execute() const;

  int dev = -1;
  int64_t count = 0;
  int flags = 0;
  bool solve_only = false;
  bool use_graph = true;
  bool ext_factors = false;
  bool lookahead = false;  // overlap the next panels with the current update (from step 1 on)
  int lookahead_mode = -1;  // set before build: -1 automatic (orders above 512), 0 off, 1 on
  cudaStream_t alloc_stream = nullptr;  // stream-ordered allocations (freed on it too)
  int64_t a_elems = 0, b_elems = 0, inv_elems = 0, lu_elems = 0, piv_elems = 0;
  std::vector<WarpClass> warp_classes;
  std::vector<Chain> chains;
  int nchains = 3;
  int64_t nstep_sys = 0, nback = 0;
  int step_nmax = 0;
  double step_flops = 0.0, step_bytes = 0.0;

  SysDesc* d_desc = nullptr;
  int32_t* d_order = nullptr;
  int32_t* d_step_list = nullptr;
  StepItem* d_items = nullptr;
  StepItem* d_back = nullptr;
  StepScratch* d_scratch = nullptr;
  double* d_lu = nullptr;
  int32_t* d_piv = nullptr;

  // device staging for host-buffer execution, allocated on first use
  double *hA = nullptr, *hB = nullptr, *hX = nullptr, *hInv = nullptr, *hDet = nullptr,
         *hSign = nullptr, *hLog = nullptr;
  int32_t* hInfo = nullptr;

 private:
  void add_cost(const SysDesc& s, double& fl, double& by) const;
  cudaError_t ensure_lookahead();  // a side stream and two events per chain
  // forward (getrs) or back substitution of one chain's strips
  cudaError_t substitute(const StepArgs& sa, const Chain& ch, cudaStream_t st, bool forward) const;
  Batch warp_batch(const Ptrs& p) const;
  StepArgs step_args(const Ptrs& p) const;

  std::mutex mu;
  Ptrs key{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;
  std::vector<cudaStream_t> side;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaEvent_t done = nullptr;  // end of the last execution: the next one waits for it
  std::vector<cudaStream_t> la_side;  // per chain: the look-ahead's other strips
  std::vector<cudaEvent_t> la_first, la_rest;
};

// A cached plan for `count` systems of order n (uniform layout), for the
// uniform-batch entry points.
std::shared_ptr<Plan> uniform_plan(int64_t count, int32_t n, int32_t nrhs, int flags, bool solve_only,
                                   bool own_lu, int* rc);

}  // namespace nppb
