// Cooperative (warp-per-quartet) ERI kernel: per-class program metadata and launch API.
#pragma once
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

}  // namespace gbx
