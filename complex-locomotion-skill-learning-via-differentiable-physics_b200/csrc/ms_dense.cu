// ms_dense.cu -- the batched-controller kernels (ms_dense.cuh) and their
// launches, compiled into their own module (see ms_dense_host.h).
#include <algorithm>
#include <type_traits>

#include "ms_dense.cuh"
#include "ms_dense_host.h"

// threads of the step kernels (one CTA per env)
#ifndef CLS_STEP_THREADS
#define CLS_STEP_THREADS 128
#endif

namespace cls {

template <typename R>
int DenseLaunch<R>::tile_m() { return std::is_same<R, float>::value ? umma::TM : kSimtTile; }
template <typename R>
int DenseLaunch<R>::tile_n() { return std::is_same<R, float>::value ? kDenseTN : kSimtTile; }
template <typename R>
long long DenseLaunch<R>::split_floats(int rows, int tile_rows, int k) {
  return (long long)umma::split_tiles_floats(rows, tile_rows, k);
}

template <typename R>
cudaError_t DenseLaunch<R>::setup(int threads, size_t* fwd_static, size_t* rev_static, int optin) {
  if (threads != CLS_STEP_THREADS) return cudaErrorInvalidValue;
  auto fwd = ms_step_fwd_kernel<R, CLS_STEP_THREADS>;
  auto rev = ms_step_rev_kernel<R, CLS_STEP_THREADS>;
  cudaFuncAttributes fa{}, ra{};
  cudaError_t e = cudaFuncGetAttributes(&fa, fwd);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&ra, rev);
  if (e != cudaSuccess) return e;
  *fwd_static = fa.sharedSizeBytes;
  *rev_static = ra.sharedSizeBytes;
  e = cudaFuncSetAttribute(fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)((size_t)optin - fa.sharedSizeBytes));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(rev, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)((size_t)optin - ra.sharedSizeBytes));
  if constexpr (std::is_same<R, float>::value) {
    const int sm = (int)umma::BulkShape<kDenseTN, kBulkStages>::kSmemBytes;
    if (e == cudaSuccess) e = cudaFuncSetAttribute(ms_ctrl_gemm_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(ms_ctrl_gemm_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(ms_wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  }
  return e;
}

template <typename R>
void DenseLaunch<R>::step_fwd(const MsArgs<R>& a, int grid, int threads, size_t smem, cudaStream_t s, int t,
                              int t_first, int t_end, int mode, int src_slot, int k_prev, int k_cur) {
  ms_step_fwd_kernel<R, CLS_STEP_THREADS><<<grid, threads, smem, s>>>(a, t, t_first, t_end, mode, src_slot,
                                                                       k_prev, k_cur);
}

template <typename R>
void DenseLaunch<R>::step_rev(const MsArgs<R>& a, int grid, int threads, size_t smem, cudaStream_t s, int t_post,
                              int t_pre, int t_begin, int t_end, int last_seg) {
  ms_step_rev_kernel<R, CLS_STEP_THREADS><<<grid, threads, smem, s>>>(a, t_post, t_pre, t_begin, t_end,
                                                                       last_seg);
}

template <typename R>
void DenseLaunch<R>::gemm(const MsArgs<R>& a, bool adjoint, int n_jobs, const DenseJob* jobs, int kslot,
                          cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value) {
    const size_t sm = umma::BulkShape<kDenseTN, kBulkStages>::kSmemBytes;
    if (adjoint) ms_ctrl_gemm_tc_kernel<1><<<n_jobs, umma::kBulkThreads, sm, s>>>(a, jobs, kslot);
    else ms_ctrl_gemm_tc_kernel<0><<<n_jobs, umma::kBulkThreads, sm, s>>>(a, jobs, kslot);
  } else {
    if (adjoint) ms_ctrl_gemm_simt_kernel<R, 1><<<n_jobs, 256, 0, s>>>(a, jobs, kslot);
    else ms_ctrl_gemm_simt_kernel<R, 0><<<n_jobs, 256, 0, s>>>(a, jobs, kslot);
  }
}

template <typename R>
void DenseLaunch<R>::pack_weights(const R* w, R* wt, R* tiles, const TransSeg* tsegs, int n_tsegs, int n_ttiles,
                                  const SplitSeg* ssegs, int n_ssegs, long long split_total, cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value) {
    if (split_total == 0) return;
    const int blocks = (int)std::min<long long>(4096, (split_total + 255) / 256);
    ms_split_weights_kernel<<<blocks, 256, 0, s>>>(w, tiles, ssegs, n_ssegs, split_total);
  } else {
    if (n_ttiles == 0) return;
    ms_transpose_weights_kernel<R><<<n_ttiles, 256, 0, s>>>(w, wt, tsegs, n_tsegs);
  }
}

template <typename R>
void DenseLaunch<R>::wgrad(const MsArgs<R>& a, int grid_x, int n_cols, int slot0, int nslots, const WgTrans* trans,
                           const WgCol* cols, int n_jobs, const WgJob* jobs, R* gw, R* gb, cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value) {
    if (n_cols > 0 && nslots > 0)
      ms_wgrad_transpose_kernel<<<dim3(grid_x, n_cols, (nslots + kWgSlots - 1) / kWgSlots), 256, 0, s>>>(
          a, trans, cols, slot0, nslots);
    if (n_jobs > 0)
      ms_wgrad_tc_kernel<<<n_jobs, umma::kBulkThreads, umma::BulkShape<kDenseTN, kBulkStages>::kSmemBytes, s>>>(
          a, jobs, nslots, gw, gb);
  }
}

template struct DenseLaunch<float>;
template struct DenseLaunch<double>;

}  // namespace cls
