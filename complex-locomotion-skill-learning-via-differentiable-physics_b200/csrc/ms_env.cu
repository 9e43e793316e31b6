// ms_env.cu -- one substep of every env with actuations chosen outside the
// library: the environment step of an external policy (a reinforcement-
// learning agent driving MassSpringEnv.step, multitask/mass_spring_env.py:55-93,
// instead of the embedded controller).  Per call and env: the given outputs
// drive apply_spring_force and advance_toi of substep t - 1
// (solver_mass_spring.py:86-148), then compute_center / compute_height and
// nn_input of t (solver_mass_spring.py:150-192, taichi_env.py:149-183) give the
// observation row in the reference's layout.  The state stays on the device
// between calls (live_x / live_v).  Compiled into its own module, like the
// batched-controller kernels, so that the fused segment kernels' module is
// unchanged.
#include <cuda_runtime.h>

#include "ms_env_host.h"
#include "ms_segment.cuh"

namespace cls {

constexpr int kEnvThreads = 128;

// One CTA per env (internal order).  outs: [n_envs][out_pitch] outputs of
// substep t - 1, or null to observe the state at t (taken from checkpoint
// slot 0 when from_ckpt).  obs: [n_envs][obs_pitch] rows in the reference's
// input layout; aux: [n_envs][4] = centre, height of t.
template <typename R>
__global__ void __launch_bounds__(kEnvThreads)
ms_env_step_kernel(MsArgs<R> a, int t, int from_ckpt, const R* __restrict__ outs, int out_pitch,
                   R* __restrict__ obs, int obs_pitch, R* __restrict__ aux) {
  extern __shared__ __align__(256) char smem_raw[];
  __shared__ RobotDesc rb;
  __shared__ EnvDesc ed;
  const int e = blockIdx.x;
  if (e >= a.n_envs) return;
  FwdSmem<R> s = carve_fwd<R>(smem_raw, a);
  const int tid = threadIdx.x, nt = blockDim.x;
  load_descs<R>(a, e, rb, ed);
  const int N = rb.n_v;
  {
    const V4<R>* cx = (from_ckpt ? a.ckpt_x : a.live_x) + ed.v_off;
    const V4<R>* cv = (from_ckpt ? a.ckpt_v : a.live_v) + ed.v_off;
    for (int i = tid; i < N; i += nt) { s.xs[i] = cx[i]; s.vs[i] = cv[i]; }
  }
  __syncthreads();
  if (outs) {
    const R* o = outs + (size_t)e * out_pitch;
    for (int q = tid; q < rb.n_out; q += nt) s.buf0[q] = o[q];
    __syncthreads();
    fwd_post<R>(a, rb, ed, s, t - 1, FWD_OBS, 0, s.buf0);
  }
  R hprev = (t > 0) ? a.obs_height[(size_t)(t - 1) * a.n_envs + e] : R(0);
  load_head_smem<R>(a, rb, ed, s, t, FWD_OBS);
  fwd_pre<R>(a, rb, ed, s, e, t, 0, FWD_OBS, 0, false, false, hprev);
  // the observation row in the reference's layout: n_sin sines, then per
  // vertex (x - c) / 0.2 and three zero velocity slots, then the goal values
  // repeated duplicate_v (vx, vz pairs), duplicate_h and duplicate_c times
  R* ob = obs + (size_t)e * obs_pitch;
  const int ns = a.n_sin, p0 = rb.pos_pad;
  const int base = ns + 6 * N;
  const int n_in = base + 2 * a.dup_v + a.dup_h + a.dup_c;
  for (int q = tid; q < n_in; q += nt) {
    R v = 0;
    if (q < ns) {
      v = s.ain[p0 + q];
    } else if (q < base) {
      const int i = (q - ns) / 6, d = (q - ns) % 6;
      v = d < 3 ? s.ain[3 * i + d] : R(0);
    } else {
      int g = q - base, col;
      if (g < 2 * a.dup_v) {
        col = g & 1;
      } else {
        g -= 2 * a.dup_v;
        const int gv = a.dup_v > 0 ? 2 : 0;
        col = g < a.dup_h ? gv : gv + (a.dup_h > 0 ? 1 : 0);
      }
      v = s.ain[p0 + ns + col];
    }
    ob[q] = v;
  }
  if (tid == 0) {
    const size_t o = (size_t)t * a.n_envs + e;
    const V4<R> c = a.obs_center[o];
    aux[4 * e] = c.x;
    aux[4 * e + 1] = c.y;
    aux[4 * e + 2] = c.z;
    aux[4 * e + 3] = a.obs_height[o];
  }
  for (int i = tid; i < N; i += nt) {
    a.live_x[ed.v_off + i] = s.xs[i];
    a.live_v[ed.v_off + i] = s.vs[i];
  }
}

template <typename R>
cudaError_t EnvLaunch<R>::step(const MsArgs<R>& a, size_t smem, cudaStream_t s, int t, int from_ckpt,
                               const R* outs, int out_pitch, R* obs, int obs_pitch, R* aux) {
  auto fn = ms_env_step_kernel<R>;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa{};
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  if (smem + fa.sharedSizeBytes > (size_t)optin) return cudaErrorInvalidConfiguration;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fn<<<a.n_envs, kEnvThreads, smem, s>>>(a, t, from_ckpt, outs, out_pitch, obs, obs_pitch, aux);
  return cudaGetLastError();
}

template struct EnvLaunch<float>;
template struct EnvLaunch<double>;

}  // namespace cls
