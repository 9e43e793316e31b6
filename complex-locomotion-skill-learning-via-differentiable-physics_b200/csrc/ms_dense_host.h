// ms_dense_host.h -- host-side launch interface of the batched-controller
// kernels (csrc/ms_dense.cu).  Those kernels live in their own translation
// unit, hence their own module: instantiated in the same module as the fused
// segment kernels, they slowed the fused reverse kernel by 10 % without ever
// being launched (measured on the 512-robot uneven batch).
#pragma once
#include <cuda_runtime.h>

#include "ms_kernels.cuh"

namespace cls {

template <typename R>
struct DenseLaunch {
  // GEMM tile of one job (envs x outputs): tensor-core tile for FP32, SIMT for FP64
  static int tile_m();
  static int tile_n();
  // floats of a pre-split operand (rows x k) in tiles of tile_rows rows (FP32)
  static long long split_floats(int rows, int tile_rows, int k);
  // shared-memory attributes of the step and GEMM kernels; the step kernels'
  // static shared bytes are returned for the capacity check
  static cudaError_t setup(int threads, size_t* fwd_static, size_t* rev_static, int optin);
  static void step_fwd(const MsArgs<R>& a, int grid, int threads, size_t smem, cudaStream_t s, int t, int t_first,
                       int t_end, int mode, int src_slot, int k_prev, int k_cur);
  static void step_rev(const MsArgs<R>& a, int grid, int threads, size_t smem, cudaStream_t s, int t_post,
                       int t_pre, int t_begin, int t_end, int last_seg);
  static void gemm(const MsArgs<R>& a, bool adjoint, int n_jobs, const DenseJob* jobs, int kslot, cudaStream_t s);
  // FP32 weight-gradient products of record slots [slot0, slot0 + nslots):
  // record transposes (grid grid_x x n_cols x slot groups) then the tensor-core
  // tiles (n_jobs CTAs), adding into gw / gb
  static void wgrad(const MsArgs<R>& a, int grid_x, int n_cols, int slot0, int nslots, const WgTrans* trans,
                    const WgCol* cols, int n_jobs, const WgJob* jobs, R* gw, R* gb, cudaStream_t s);
  // FP32: W_l and W_l^T as pre-split tiles; FP64: W_l^T
  static void pack_weights(const R* w, R* wt, R* tiles, const TransSeg* tsegs, int n_tsegs, int n_ttiles,
                           const SplitSeg* ssegs, int n_ssegs, long long split_total, cudaStream_t s);
};

}  // namespace cls
