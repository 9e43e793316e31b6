// ms_env_host.h -- host-side launch interface of the external-policy
// environment step (csrc/ms_env.cu, its own module).
#pragma once
#include <cuda_runtime.h>

#include "ms_kernels.cuh"

namespace cls {

template <typename R>
struct EnvLaunch {
  // one substep of every env (a.n_envs CTAs); see ms_env_step_kernel
  static cudaError_t step(const MsArgs<R>& a, size_t smem, cudaStream_t s, int t, int from_ckpt, const R* outs,
                          int out_pitch, R* obs, int obs_pitch, R* aux);
};

}  // namespace cls
