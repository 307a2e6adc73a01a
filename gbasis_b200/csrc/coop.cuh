// Cooperative (warp-per-quartet) ERI kernel: per-class program metadata and launch API.
#pragma once
#include <vector>

#include "gbx_common.cuh"

namespace gbx {

// Offsets (into kCoopIns / kCoopLv / kCoopIdx) and sizes of one class's programs.
struct CoopMeta {
  int la, lb, lc, ld, L, NE, NF, nX, nK, nB;
  int v_ins, v_lv, v_nlv, t_ins, t_lv, t_nlv, k_ins, k_lv, k_nlv, b_ins, b_lv, b_nlv;
  int targets, kfin, bfin;
  int n_ins, n_idx;  // instructions (VRR, ETR, ket, bra programs, contiguous) and indices
};

// Find the program of class (la, lb | lc, ld); -1 when the class is not cooperative.
int coop_class(int la, int lb, int lc, int ld);
int launch_coop(int prog, const EriLaunch& a, cudaStream_t st);

// Multi-class work queue (eri_queue): one persistent launch drains the quartets of many class
// blocks (or batch block types) from a single queue.  Segment k holds queue positions
// [first, first + n): the quartets work[work_off + i], i < n, of launches[k]'s block.
struct QueueSeg {
  long long first, n;
};
struct QueuePlan {
  int nseg = 0;
  long long total = 0;      // quartets in the queue
  int smem_per_warp = 0;    // doubles: the largest segment's need
  int wpc = 1;              // warps per CTA
  size_t smem = 0;          // dynamic shared memory per CTA
  size_t args_bytes = 0;    // bytes of the per-segment argument table (queue_plan's blob)
};
// Program of any class, light or heavy, for the queue kernel; -1 when none was generated.
int coop_program(int la, int lb, int lc, int ld);
// Per-segment launch arguments of the queue (programs read from the global tables, tail
// chunking per class within the launch's shared memory) as a blob to upload, and the plan.
// launches[k]: the block's arguments (work list, store, mode 0); progs[k]: coop_program.
int queue_plan(const EriLaunch* launches, const int* progs, const long long* counts, int nseg,
               std::vector<unsigned char>& args_blob, std::vector<QueueSeg>& segs,
               QueuePlan& plan);
// One persistent launch over the queue; *cursor must be zero (the kernel draws from it).
int launch_queue(const void* d_args, const QueueSeg* d_segs, unsigned long long* cursor,
                 const QueuePlan& plan, int device, cudaStream_t st);

}  // namespace gbx
