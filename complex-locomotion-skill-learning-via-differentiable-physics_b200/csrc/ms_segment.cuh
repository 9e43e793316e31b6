// ms_segment.cuh -- segment kernels: forward (first pass / recompute), reverse,
// losses, weight-gradient products, Adam and weight packing.
#pragma once
#include "ms_kernels.cuh"

namespace cls {

// FWD_RECTAIL (first pass of an episode of several segments): substeps from
// MsArgs::rec_from on are recorded at slot t - rec_from, as the last
// segment's recompute would record them, so the reverse pass starts without
// that recompute.
// FWD_RECCTRL (first pass, whole-episode controller records): the controller
// records (input, pre-activations) of every substep at slot t.
// FWD_REPLAY (recompute over those records): the controller outputs of each
// substep come from its recorded output-layer pre-activations (the same
// values, so the same state bit for bit) instead of the inputs and products.
enum FwdMode : int {
  FWD_CKPT = 1, FWD_OBS = 2, FWD_RECORD = 4, FWD_CKEND = 8, FWD_RECTAIL = 16, FWD_RECCTRL = 32, FWD_REPLAY = 64
};

// episode steps of env e (per-env in served batches)
template <typename R>
__device__ __forceinline__ int steps_of(const MsArgs<R>& a, int e) {
  return a.env_steps ? a.env_steps[e] : a.steps;
}

// sum of M values over the block, deterministic; red must hold 32*M entries
template <typename R, int M>
__device__ __forceinline__ void block_sum(R (&v)[M], R* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int m = 0; m < M; ++m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[m] += __shfl_xor_sync(0xffffffffu, v[m], o);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) red[m * 32 + wid] = v[m];
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < M; ++m) {
    R s = 0;
    for (int w = 0; w < nw; ++w) s += red[m * 32 + w];
    v[m] = s;
  }
  __syncthreads();
}

// min (or max) of y with the LAST index attaining it, over the block
template <typename R>
__device__ __forceinline__ void block_argext(R& val, int& idx, bool is_min, R* red, int* redi) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  auto better = [&](R v1, int i1, R v2, int i2) {  // is (v2,i2) preferred over (v1,i1)?
    if (is_min) return (v2 < v1) || (v2 == v1 && i2 > i1);
    return (v2 > v1) || (v2 == v1 && i2 > i1);
  };
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    R v2 = __shfl_xor_sync(0xffffffffu, val, o);
    int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
    if (better(val, idx, v2, i2)) { val = v2; idx = i2; }
  }
  __syncthreads();
  if (lane == 0) { red[wid] = val; redi[wid] = idx; }
  __syncthreads();
  R bv = red[0];
  int bi = redi[0];
  for (int w = 1; w < nw; ++w)
    if (better(bv, bi, red[w], redi[w])) { bv = red[w]; bi = redi[w]; }
  val = bv;
  idx = bi;
  __syncthreads();
}

template <typename R>
__device__ __forceinline__ void load_descs(const MsArgs<R>& a, int e, RobotDesc& rb, EnvDesc& ed) {
  // cooperative word copy of the two small descriptors into shared memory
  const int* se = reinterpret_cast<const int*>(a.envs + e);
  int* de = reinterpret_cast<int*>(&ed);
  for (int q = threadIdx.x; q < (int)(sizeof(EnvDesc) / 4); q += blockDim.x) de[q] = se[q];
  __syncthreads();
  const int* sr = reinterpret_cast<const int*>(a.robots + ed.robot);
  int* dr = reinterpret_cast<int*>(&rb);
  for (int q = threadIdx.x; q < (int)(sizeof(RobotDesc) / 4); q += blockDim.x) dr[q] = sr[q];
  __syncthreads();
}

// goal columns of the compact input: (vx, vz) / max_speed if duplicate_v > 0,
// target height if duplicate_h > 0, crawl target if duplicate_c > 0
// The observables' reductions of one substep in one pass: sums v[0..10]
// (centre, then the heading sides' coordinate sums and counts) in block_sum's
// order, and the min / max of the height with block_argext's order -- the same
// bits as block_sum<R, 3> + 2 x block_argext + block_sum<R, 8>, with two
// barriers instead of ten.  red: kRedFwd entries (sums at [m * 32 + warp], the
// extrema at [352 + warp] and [384 + warp], their indices as ints from 416).
template <typename R>
__device__ __forceinline__ void block_obs(R (&v)[11], R& lo, int& li, R& hi, int& hidx, R* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int* redi = reinterpret_cast<int*>(red + 416);
#pragma unroll
  for (int m = 0; m < 11; ++m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[m] += __shfl_xor_sync(0xffffffffu, v[m], o);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const R l2 = __shfl_xor_sync(0xffffffffu, lo, o);
    const int li2 = __shfl_xor_sync(0xffffffffu, li, o);
    if ((l2 < lo) || (l2 == lo && li2 > li)) { lo = l2; li = li2; }
    const R h2 = __shfl_xor_sync(0xffffffffu, hi, o);
    const int hi2 = __shfl_xor_sync(0xffffffffu, hidx, o);
    if ((h2 > hi) || (h2 == hi && hi2 > hidx)) { hi = h2; hidx = hi2; }
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int m = 0; m < 11; ++m) red[m * 32 + wid] = v[m];
    red[352 + wid] = lo;
    red[384 + wid] = hi;
    redi[wid] = li;
    redi[32 + wid] = hidx;
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < 11; ++m) {
    R sm = 0;
    for (int w = 0; w < nw; ++w) sm += red[m * 32 + w];
    v[m] = sm;
  }
  lo = red[352]; li = redi[0];
  hi = red[384]; hidx = redi[32];
  for (int w = 1; w < nw; ++w) {
    const R l2 = red[352 + w], h2 = red[384 + w];
    const int li2 = redi[w], hi2 = redi[32 + w];
    if ((l2 < lo) || (l2 == lo && li2 > li)) { lo = l2; li = li2; }
    if ((h2 > hi) || (h2 == hi && hi2 > hidx)) { hi = h2; hidx = hi2; }
  }
}

// Heading sides of the env's vertices (set at t = 0 by the first pass) into
// shared memory, for a range that starts after t = 0; the vertex-to-thread
// mapping is the one fwd_pre reads them with.
template <typename R>
__device__ __forceinline__ void load_head_smem(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                               const FwdSmem<R>& s, int t, int mode) {
  if (!(mode & FWD_OBS) || t == 0 || rb.robot_id == 100) return;
  for (int i = threadIdx.x; i < rb.n_v; i += blockDim.x) s.head[i] = a.head[ed.v_off + i];
}

template <typename R>
__device__ __forceinline__ R goal_value(const MsArgs<R>& a, int g, size_t o) {
  if (a.dup_v > 0) {
    if (g == 0) return a.tv[o].x / a.max_speed;
    if (g == 1) return a.tv[o].z / a.max_speed;
    g -= 2;
  }
  if (a.dup_h > 0) {
    if (g == 0) return a.th[o];
    g -= 1;
  }
  if (a.dup_c > 0 && g == 0) return a.tc[o];
  return R(0);
}

template <typename R>
__device__ __forceinline__ int next_item(const MsArgs<R>& a, int* s_item) {
  if (threadIdx.x == 0) *s_item = atomicAdd(a.queue, 1);
  __syncthreads();
  int it = *s_item;
  __syncthreads();
  return it;
}

// ---------------------------------------------------------------- forward
// The two halves of one substep around the controller, shared by the fused
// segment kernel (MLP in between, per env) and the batched-controller step
// kernels (MLP as tensor-core GEMMs over all envs of a robot type).

// Substep t up to the controller input: checkpoint / records / trajectory of
// x(t), compute_center / compute_height / compute_rotation
// (solver_mass_spring.py:150-192) into the observables, nn_input
// (taichi_env.py:149-183) into s.ain (compact column order, zero padded to
// pitch 0).  The input row is recorded at slot kslot when `rec_in` (FWD_RECORD
// or the batched path, which also records the zero padding).  hprev: running
// height of t - 1, updated to t.
template <typename R>
__device__ __forceinline__ void fwd_pre(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                        const FwdSmem<R>& s, int e, int t, int t_begin, int mode,
                                        int kslot, bool rec_in, bool rec_pad, R& hprev, int kc = -1) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int N = rb.n_v;
  const R invN = R(1) / R(N);
  if ((mode & FWD_CKPT) && t > t_begin && (t % a.K) == 0) {
    V4<R>* cx = a.ckpt_x + (size_t)(t / a.K) * a.v_total + ed.v_off;
    V4<R>* cv = a.ckpt_v + (size_t)(t / a.K) * a.v_total + ed.v_off;
    bool bad = false;
    for (int i = tid; i < N; i += nt) {
      cx[i] = s.xs[i]; cv[i] = s.vs[i];
      bad |= !(finite(s.xs[i].x) && finite(s.xs[i].y) && finite(s.xs[i].z));
    }
    if (bad) atomicOr(a.status, ERR_NONFINITE);
  }
  if (mode & FWD_RECORD) {
    V4<R>* rx = a.rec_x + (size_t)kslot * a.v_total + ed.v_off;
    V4<R>* rv = a.rec_v + (size_t)kslot * a.v_total + ed.v_off;
    for (int i = tid; i < N; i += nt) { rx[i] = s.xs[i]; rv[i] = s.vs[i]; }
  }
  if ((mode & FWD_OBS) && a.x_full) {
    V4<R>* xf = a.x_full + (size_t)t * a.v_total + ed.v_off;
    for (int i = tid; i < N; i += nt) xf[i] = s.xs[i];
  }
  // the goal and sine columns of the input do not depend on the state: their
  // loads are issued here and stored after the reductions
  const int p0 = rb.pos_pad, nc = rb.n_c;
  const int qpre = p0 + tid;
  R pre = 0;
  if (qpre < nc)
    pre = (qpre < p0 + a.n_sin) ? a.sin_table[(size_t)t * a.n_sin + (qpre - p0)]
                                : goal_value<R>(a, qpre - p0 - a.n_sin, (size_t)t * a.n_envs + e);
  R c[3] = {0, 0, 0};
  if ((mode & FWD_OBS) && (rb.robot_id == 100 || t > 0)) {
    // compute_center / compute_height / upper height / compute_rotation
    // (solver_mass_spring.py:150-192) in one reduction (heading sides fixed)
    const bool heading = rb.robot_id != 100;
    R v[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    R lo = R(10), hi = R(-10);
    int li = 0, hiidx = 0;
    for (int i = tid; i < N; i += nt) {
      const V4<R> p = s.xs[i];
      v[0] += p.x * invN; v[1] += p.y * invN; v[2] += p.z * invN;
      lo = fmin(lo, p.y); hi = fmax(hi, p.y);
      if (heading) {
        if (s.head[i]) { v[3] += p.x; v[4] += p.y; v[5] += p.z; v[6] += R(1); }
        else { v[7] += p.x; v[8] += p.y; v[9] += p.z; v[10] += R(1); }
      }
    }
    block_obs<R>(v, lo, li, hi, hiidx, s.red);
    c[0] = v[0]; c[1] = v[1]; c[2] = v[2];
    R rot;
    if (heading) {
      const R d0 = -v[3] * v[10] + v[7] * v[6];
      const R d2 = -v[5] * v[10] + v[9] * v[6];
      rot = datan2<R>(d2, d0);
    } else {
      R d0 = 0, d2 = 0;
      if (tid == 0) {
        const V4<R> p = s.xs[rb.rot_idx[0]], q = s.xs[rb.rot_idx[1]];
        const V4<R> u = s.xs[rb.rot_idx[2]], w = s.xs[rb.rot_idx[3]];
        d0 = p.x + q.x - u.x - w.x;
        d2 = p.z + q.z - u.z - w.z;
      }
      rot = datan2<R>(d2, d0);
    }
    // every thread holds the same lo and hprev: no broadcast
    const R h = (t % a.jump_period == 0) ? lo : fmax(hprev, lo);
    if (tid == 0) {
      const size_t o = (size_t)t * a.n_envs + e;
      V4<R> cc; cc.x = c[0]; cc.y = c[1]; cc.z = c[2]; cc.w = 0;
      a.obs_center[o] = cc;
      a.obs_height[o] = h;
      a.obs_upper[o] = hi;
      a.obs_rot[o] = rot;
    }
    hprev = h;
  } else {
    // -- compute_center (solver_mass_spring.py:150-156): sum of x / n
    for (int i = tid; i < N; i += nt) {
      c[0] += s.xs[i].x * invN; c[1] += s.xs[i].y * invN; c[2] += s.xs[i].z * invN;
    }
    block_sum<R, 3>(c, s.red);
    if (mode & FWD_OBS) {
      // t = 0, heading sides from the centre: compute_height / upper height
      // (solver_mass_spring.py:158-173), compute_rotation (:175-192)
      R lo = R(10), hi = R(-10);
      for (int i = tid; i < N; i += nt) { lo = fmin(lo, s.xs[i].y); hi = fmax(hi, s.xs[i].y); }
      int li = 0, hiidx = 0;
      block_argext<R>(lo, li, true, s.red, reinterpret_cast<int*>(s.red + kRedInt));
      block_argext<R>(hi, hiidx, false, s.red, reinterpret_cast<int*>(s.red + kRedInt));
      unsigned char* hd = a.head + ed.v_off;
      for (int i = tid; i < N; i += nt) {
        const unsigned char f = (s.xs[i].x < c[0]) ? 1 : 0;
        hd[i] = f;
        s.head[i] = f;
      }
      R hs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int i = tid; i < N; i += nt) {
        const V4<R> p = s.xs[i];
        if (s.head[i]) { hs[0] += p.x; hs[1] += p.y; hs[2] += p.z; hs[3] += R(1); }
        else { hs[4] += p.x; hs[5] += p.y; hs[6] += p.z; hs[7] += R(1); }
      }
      block_sum<R, 8>(hs, s.red);
      const R d0 = -hs[0] * hs[7] + hs[4] * hs[3];
      const R d2 = -hs[2] * hs[7] + hs[6] * hs[3];
      const R rot = datan2<R>(d2, d0);
      const R h = (t % a.jump_period == 0) ? lo : fmax(hprev, lo);
      if (tid == 0) {
        const size_t o = (size_t)t * a.n_envs + e;
        V4<R> cc; cc.x = c[0]; cc.y = c[1]; cc.z = c[2]; cc.w = 0;
        a.obs_center[o] = cc;
        a.obs_height[o] = h;
        a.obs_upper[o] = hi;
        a.obs_rot[o] = rot;
      }
      hprev = h;
    }
  }
  // -- nn_input (taichi_env.py:149-183) in the compact column order
  {
    const int pitch0 = rb.pitch[0];
    const int nrec = rec_pad ? pitch0 : nc;
    R* rin = rec_in ? a.rec_in + (size_t)(kc >= 0 ? kc : kslot) * a.in_total + ed.in_off : nullptr;
    for (int q = tid; q < pitch0; q += nt) {
      if (q >= p0 && q < nc && q - p0 < nt) continue;  // loaded ahead (pre)
      R val = 0;
      if (q < 3 * N) {
        const int i = q / 3, d = q - 3 * (q / 3);
        val = (comp(s.xs[i], d) - c[d]) / R(0.2);
      } else if (q >= p0 && q < p0 + a.n_sin) {
        val = a.sin_table[(size_t)t * a.n_sin + (q - p0)];
      } else if (q >= p0 + a.n_sin && q < nc) {
        val = goal_value<R>(a, q - p0 - a.n_sin, (size_t)t * a.n_envs + e);
      }
      s.ain[q] = val;
      if (rin && q < nrec) rin[q] = val;
    }
    if (qpre < nc) {
      s.ain[qpre] = pre;
      if (rin && qpre < nrec) rin[qpre] = pre;
    }
  }
  __syncthreads();
}

// Substep t after the controller: actuation record, apply_spring_force
// (gather form) with the controller outputs `out`, advance_toi.
template <typename R>
__device__ __forceinline__ void fwd_post(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                         const FwdSmem<R>& s, int t, int mode, int kslot, const R* out) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int N = rb.n_v, L = rb.n_layers;
  if ((mode & FWD_OBS) && a.act_full) {
    R* af = a.act_full + (size_t)t * a.z_total[L - 1] + ed.z_off[L - 1];
    for (int o = tid; o < rb.n_out; o += nt) af[o] = out[o];
  }
  V4<R>* rec = (mode & FWD_RECORD) ? a.rec_vinc + (size_t)kslot * a.v_total + ed.v_off : nullptr;
  if (s.imp)
    gather_vinc_table<R>(a, rb, N, s.xs, s.vs, out, s.imp, s.vinc, rec);
  else
    gather_vinc_all<R>(a, rb, N, s.xs, s.vs, out, s.vinc, rec);
  __syncthreads();
  for (int i = tid; i < N; i += nt) advance_vertex<R>(a, s.xs[i], s.vs[i], s.vinc[i]);
  __syncthreads();
}

// State after the last processed step of a range ending at t_end.
template <typename R>
__device__ __forceinline__ void fwd_finish(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                           const FwdSmem<R>& s, int t_begin, int t_end, int mode) {
  const int tid = threadIdx.x, nt = blockDim.x, N = rb.n_v;
  if ((mode & FWD_CKEND) && t_end % a.K == 0 && t_end > t_begin) {
    V4<R>* cx = a.ckpt_x + (size_t)(t_end / a.K) * a.v_total + ed.v_off;
    V4<R>* cv = a.ckpt_v + (size_t)(t_end / a.K) * a.v_total + ed.v_off;
    for (int i = tid; i < N; i += nt) { cx[i] = s.xs[i]; cv[i] = s.vs[i]; }
  }
  if (mode & FWD_OBS) {
    for (int i = tid; i < N; i += nt) {
      a.fin_x[ed.v_off + i] = s.xs[i];
      a.fin_v[ed.v_off + i] = s.vs[i];
    }
    if (a.x_full && t_end < a.T) {
      V4<R>* xf = a.x_full + (size_t)t_end * a.v_total + ed.v_off;
      for (int i = tid; i < N; i += nt) xf[i] = s.xs[i];
    }
  }
  __syncthreads();
}

// Advances every env from t_begin (state in checkpoint slot src_slot) through
// t_end (exclusive), i.e. runs pre_advance/nn_input/forward/advance for each t.
template <typename R, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
ms_forward_kernel(MsArgs<R> a, int t_begin0, int t_end0, int mode, int src_slot0) {
  extern __shared__ __align__(256) char smem_raw[];
  __shared__ RobotDesc rb;
  __shared__ EnvDesc ed;
  __shared__ int s_item;
  FwdSmem<R> s = carve_fwd<R>(smem_raw, a);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (;;) {
    const int item = next_item(a, &s_item);
    if (item >= a.n_items) break;
    const int e = a.order[item];
    int t_begin = t_begin0, t_end = t_end0, src_slot = src_slot0;
    if (a.win) {
      const int4 w = a.win[e];
      t_begin = w.x; t_end = w.y; src_slot = w.z;
    }
    load_descs(a, e, rb, ed);
    const int N = rb.n_v, L = rb.n_layers;
    {
      const V4<R>* cx = a.ckpt_x + (size_t)src_slot * a.v_total + ed.v_off;
      const V4<R>* cv = a.ckpt_v + (size_t)src_slot * a.v_total + ed.v_off;
      for (int i = tid; i < N; i += nt) { s.xs[i] = cx[i]; s.vs[i] = cv[i]; }
    }
    if (s.w) load_controller_smem<R>(a.w, a.bias, rb, s.w, s.b);
    load_head_smem<R>(a, rb, ed, s, t_begin, mode);
    R hprev = 0;
    if ((mode & FWD_OBS) && t_begin > 0) hprev = a.obs_height[(size_t)(t_begin - 1) * a.n_envs + e];
    __syncthreads();
    CLS_PHASE_START();
    for (int t = t_begin; t < t_end; ++t) {
      int kk = t - t_begin, mode_t = mode;
      if ((mode & FWD_RECTAIL) && t >= a.rec_from) {
        mode_t |= FWD_RECORD;
        kk = t - a.rec_from;
      }
      if (mode & FWD_REPLAY) {
        // state records of t, then the controller outputs from the recorded
        // output-layer pre-activations (act(z + b), as dense_forward forms them)
        if (mode_t & FWD_RECORD) {
          V4<R>* rx = a.rec_x + (size_t)kk * a.v_total + ed.v_off;
          V4<R>* rv = a.rec_v + (size_t)kk * a.v_total + ed.v_off;
          for (int i = tid; i < N; i += nt) { rx[i] = s.xs[i]; rv[i] = s.vs[i]; }
        }
        const int lo = L - 1, nout = rb.width[L];
        const R* zr = a.rec_z + a.z_base[lo] + (size_t)kk * a.z_total[lo] + ed.z_off[lo];
        const R* bo = s.w ? s.b + (rb.b_off[lo] - rb.b_off[0]) : a.bias + rb.b_off[lo];
        R* y = (lo & 1) ? s.buf1 : s.buf0;
        for (int o = tid; o < ((nout + 3) & ~3); o += nt) y[o] = o < nout ? act_f<R>(a.act_out, zr[o] + bo[o]) : R(0);
        __syncthreads();
        fwd_post<R>(a, rb, ed, s, t, mode_t, kk, y);
        continue;
      }
      // controller records: at slot t over the whole episode (FWD_RECCTRL),
      // else with the state records at kk
      const bool rec_ctrl = (mode_t & FWD_RECORD) || (mode & FWD_RECCTRL);
      const int kc = (mode & FWD_RECCTRL) ? t : kk;
      fwd_pre<R>(a, rb, ed, s, e, t, t_begin, mode_t, kk, rec_ctrl, false, hprev, kc);
      CLS_PHASE(a, 10);
      // -- MLP (nn.py:130-146): z = W a, a' = act(z + b)
      R* out = nullptr;
      for (int l = 0; l < L; ++l) {
        const R* in = (l == 0) ? s.ain : ((l & 1) ? s.buf0 : s.buf1);
        R* y = (l & 1) ? s.buf1 : s.buf0;
        const int nout = rb.width[l + 1];
        R* zrec = rec_ctrl ? a.rec_z + a.z_base[l] + (size_t)kc * a.z_total[l] + ed.z_off[l] : nullptr;
        const int act = l == L - 1 ? a.act_out : a.act_hidden;
        if (s.w)
          dense_forward<R, true>(s.w + (rb.w_off[l] - rb.w_off[0]), rb.pitch[l], nout,
                                 s.b + (rb.b_off[l] - rb.b_off[0]), in, y, zrec, act);
        else
          dense_forward<R, false>(a.w + rb.w_off[l], rb.pitch[l], nout, a.bias + rb.b_off[l], in, y,
                                  zrec, act);
        // zero the padding up to the next layer's pitch
        const int padto = (l + 1 < L) ? rb.pitch[l + 1] : ((nout + 3) & ~3);
        for (int q = nout + tid; q < padto; q += nt) y[q] = 0;
        __syncthreads();
        out = y;
      }
      CLS_PHASE(a, 13);
      fwd_post<R>(a, rb, ed, s, t, mode_t, kk, out);
      CLS_PHASE(a, 16);
    }
    fwd_finish<R>(a, rb, ed, s, t_begin, t_end, mode);
  }
}

// -------------------------------------------------------------- loss seeds
template <typename R>
__device__ __forceinline__ V4<R> obs_c(const MsArgs<R>& a, int t, int e) {
  return a.obs_center[(size_t)t * a.n_envs + e];
}

// d loss / d center[t] from the velocity loss (taichi_env.py:185-211)
// Its observables and targets are loaded first (load_center_velocity, before
// the block reduction of the centre adjoint, so the loads overlap it) and
// applied after (apply_center_velocity, the same expressions in the same order).
template <typename R>
struct CenterVelocitySeed {
  bool on1, on2;
  R sc;
  V4<R> c1a, c0a, tva, c1b, c0b, tvb;
};
template <typename R>
__device__ __forceinline__ CenterVelocitySeed<R> load_center_velocity(const MsArgs<R>& a, int t, int e, R Br) {
  const int rp = a.run_period, tp = a.turn_period, st = steps_of(a, e);
  CenterVelocitySeed<R> q;
  q.sc = R(2) * R(100) / R(st) / Br;
  q.on1 = (a.loss_mask & LOSS_VELOCITY) && t >= rp && t % tp > rp && t <= st && t < a.T;
  if (q.on1) {
    q.c1a = obs_c(a, t, e); q.c0a = obs_c(a, t - rp, e);
    q.tva = a.tv[(size_t)(t - rp) * a.n_envs + e];
  }
  const int u = t + rp;
  q.on2 = (a.loss_mask & LOSS_VELOCITY) && u <= st && u < a.T && u % tp > rp;
  if (q.on2) {
    q.c1b = obs_c(a, u, e); q.c0b = obs_c(a, t, e);
    q.tvb = a.tv[(size_t)t * a.n_envs + e];
  }
  return q;
}
template <typename R>
__device__ __forceinline__ void apply_center_velocity(const CenterVelocitySeed<R>& q, R g[3]) {
  if (q.on1) {
    g[0] += (q.c1a.x - q.c0a.x - q.tva.x) * q.sc;
    g[2] += (q.c1a.z - q.c0a.z - q.tva.z) * q.sc;
  }
  if (q.on2) {
    g[0] -= (q.c1b.x - q.c0b.x - q.tvb.x) * q.sc;
    g[2] -= (q.c1b.z - q.c0b.z - q.tvb.z) * q.sc;
  }
}

// d loss / d x[t, i] and d loss / d center[t] from the rotation loss
// (taichi_env.py:235-252) and pose loss (:224-233).  Adds to gxi and gc.
template <typename R>
__device__ __forceinline__ void seed_x_rotation_pose(const MsArgs<R>& a, const RobotDesc& rb,
                                                     const EnvDesc& ed, int t, int e, int i,
                                                     const V4<R>& xi, R Br, R gxi[3], R gc[3]) {
  const int rp = a.run_period, tp = a.turn_period, st = steps_of(a, e);
  if (a.loss_mask & LOSS_ROTATION) {
    const R k = R(2) / R(40) / R(st);
    if (t >= 1 && t % tp > rp && t <= st && t < a.T) {
      const V4<R> c1 = obs_c(a, t, e), c0 = obs_c(a, t - rp, e);
      const V4<R> x0 = a.x_full[(size_t)(t - rp) * a.v_total + ed.v_off + i];
      const R ang = a.th[(size_t)(t - rp) * a.n_envs + e] * R(72.) / R(180.) * R(3.1415926535);
      const R ca = dcos<R>(ang), sn = dsin<R>(ang);
      const R t0x = xi.x - c1.x, t0y = xi.y - c1.y, t0z = xi.z - c1.z;
      const R t1x = x0.x - c0.x, t1y = x0.y - c0.y, t1z = x0.z - c0.z;
      const R gx = (t0x - (ca * t1x - sn * t1z)) * k;
      const R gy = (t0y - t1y) * k;
      const R gz = (t0z - (sn * t1x + ca * t1z)) * k;
      gxi[0] += gx; gxi[1] += gy; gxi[2] += gz;
      gc[0] -= gx; gc[1] -= gy; gc[2] -= gz;
    }
    const int u = t + rp;
    if (u <= st && u < a.T && u % tp > rp) {
      const V4<R> c1 = obs_c(a, u, e), c0 = obs_c(a, t, e);
      const V4<R> x1 = a.x_full[(size_t)u * a.v_total + ed.v_off + i];
      const R ang = a.th[(size_t)t * a.n_envs + e] * R(72.) / R(180.) * R(3.1415926535);
      const R ca = dcos<R>(ang), sn = dsin<R>(ang);
      const R t0x = x1.x - c1.x, t0y = x1.y - c1.y, t0z = x1.z - c1.z;
      const R t1x = xi.x - c0.x, t1y = xi.y - c0.y, t1z = xi.z - c0.z;
      const R g2x = -(t0x - (ca * t1x - sn * t1z)) * k;
      const R g2y = -(t0y - t1y) * k;
      const R g2z = -(t0z - (sn * t1x + ca * t1z)) * k;
      const R g1x = ca * g2x + sn * g2z, g1y = g2y, g1z = -sn * g2x + ca * g2z;
      gxi[0] += g1x; gxi[1] += g1y; gxi[2] += g1z;
      gc[0] -= g1x; gc[1] -= g1y; gc[2] -= g1z;
    }
  }
  if (a.loss_mask & LOSS_POSE) {
    const int jp = a.jump_period;
    if (t >= 1 && t % jp == 0 && t <= st && t < a.T) {
      const V4<R> p = a.init_obj[ed.v_off + i];
      const R k = R(2) / R(st / jp) / Br;
      gxi[0] += (xi.x - p.x) * k; gxi[1] += (xi.y - p.y) * k; gxi[2] += (xi.z - p.z) * k;
    }
  }
}

template <typename R>
__device__ __forceinline__ R seed_height(const MsArgs<R>& a, int t, int e, R Br) {
  if (!(a.loss_mask & LOSS_HEIGHT)) return 0;
  const int jp = a.jump_period, st = steps_of(a, e);
  const size_t o = (size_t)t * a.n_envs + e;
  if (t >= 1 && t <= st && t < a.T && t % jp == jp - 1 && a.th[o] > R(0.1 + 1e-6))
    return R(2) * (a.obs_height[o] - a.th[o]) * R(100) / R(st / jp) / Br;
  return 0;
}

template <typename R>
__device__ __forceinline__ R seed_upper(const MsArgs<R>& a, int t, int e, R Br) {
  if (!(a.loss_mask & LOSS_CRAWL)) return 0;
  const int st = steps_of(a, e);
  const size_t o = (size_t)t * a.n_envs + e;
  if (t >= 1 && t <= st && t < a.T && a.tc[o] > R(1 - 1e-4)) {
    const R d = a.obs_upper[o] - R(0.1);
    if (R(0) < d) return R(2) * d * R(5) / R(st) / Br;
  }
  return 0;
}

// -------------------------------------------------------------- spring adjoint
// Adjoint of apply_spring_force(t) in gather form: each vertex's half-warp
// takes its incident springs (the CSR incidence list of the forward gather),
// recomputes each spring's adjoint and adds the part that falls on its own
// vertex, so d x and d v need no atomics and sum in a fixed order; the
// a-side incidence of an actuated spring adds d actuation (shared-memory
// atomic: outputs may drive several springs).  Twice the spring arithmetic of
// a spring-parallel adjoint, in exchange for its 12 shared-memory atomics per
// spring, which bounded that form (the reverse kernels 10-16 % faster).
// Adjoint terms of one spring's impulse (evaluated in a -> b order): gd =
// d loss / d x_a (x_b takes -gd), h = d loss / d v_a (v_b takes -h), and the
// actuation gradient's factor gact_f (d act = gact_f * coef * l0 * ...).
template <typename R>
struct SpringAdj {
  R gd0, gd1, gd2, h0, h1, h2, gact;
};
template <typename R>
__device__ __forceinline__ SpringAdj<R> spring_adjoint_terms(const MsArgs<R>& a, const V4<R>& xa, const V4<R>& xb,
                                                             const V4<R>& va, const V4<R>& vb, const V4<R>& ga,
                                                             const V4<R>& gb, R act, R l0, R k, R coef) {
  const R d0 = xa.x - xb.x, d1 = xa.y - xb.y, d2 = xa.z - xb.z;
  const R n2 = d0 * d0 + d1 * d1 + d2 * d2;
  const R r8 = sqrt_s<R>(n2 + R(1e-8));
  const R length = r8 + R(1e-4);
  const R inv_length = rcp_s<R>(length);
  const R target = l0 * (R(1) + coef * act);
  const R sc = a.dt * (length - target) * k * inv_length;
  const R invlen = rsqrt_s<R>(n2);
  const R inv_r8 = rcp_s<R>(r8);
  const R n0 = d0 * invlen, n1 = d1 * invlen, nz = d2 * invlen;
  const R dv0 = va.x - vb.x, dv1 = va.y - vb.y, dv2 = va.z - vb.z;
  const R vrel = dv0 * n0 + dv1 * n1 + dv2 * nz;
  const R gi0 = gb.x - ga.x, gi1 = gb.y - ga.y, gi2 = gb.z - ga.z;
  const R gsc = gi0 * d0 + gi1 * d1 + gi2 * d2;
  const R gvrel = a.dashpot * (gi0 * n0 + gi1 * n1 + gi2 * nz);
  const R cdv = a.dashpot * vrel;
  const R gn0 = cdv * gi0 + gvrel * dv0, gn1 = cdv * gi1 + gvrel * dv1, gn2 = cdv * gi2 + gvrel * dv2;
  SpringAdj<R> r;
  r.gd0 = sc * gi0 + invlen * gn0; r.gd1 = sc * gi1 + invlen * gn1; r.gd2 = sc * gi2 + invlen * gn2;
  const R ginv = gn0 * d0 + gn1 * d1 + gn2 * d2;
  const R gr_r = -ginv * invlen * invlen * invlen;
  r.gd0 += gr_r * d0; r.gd1 += gr_r * d1; r.gd2 += gr_r * d2;
  const R glen = gsc * a.dt * k * target * inv_length * inv_length;
  const R glen_r8 = glen * inv_r8;
  r.gd0 += glen_r8 * d0; r.gd1 += glen_r8 * d1; r.gd2 += glen_r8 * d2;
  r.h0 = gvrel * n0; r.h1 = gvrel * n1; r.h2 = gvrel * nz;
  r.gact = -gsc * a.dt * k * inv_length * l0 * coef;
  return r;
}

// d act of the spring's output, with the actuation loss's seed
// (taichi_env.py:276-285, per spring)
template <typename R>
__device__ __forceinline__ R spring_gact(R gact, R act, R act_seed_scale, R act_lim, bool act_seed) {
  if (act_seed) {
    if (R(0) < dabs<R>(act) - act_lim) gact += ((act > 0) - (act < 0)) * act_seed_scale;
  }
  return gact;
}

template <typename R>
__device__ __forceinline__ void spring_adjoint_one(const MsArgs<R>& a, const Inc<R>& in, int v,
                                                   const PairRows<R>& xv, const V4<R>* gvinc, const R* outv,
                                                   R* gout, R act_seed_scale, R act_lim, bool act_seed,
                                                   R (&gxs)[3], R (&gvs)[3]) {
  const int o = in.other;
  const int ia = in.side == 0 ? v : o, ib = in.side == 0 ? o : v;
  const R act = in.out >= 0 ? outv[in.out] : R(0);
  V4<R> xa, va, xb, vb;
  xv.get(ia, xa, va);
  xv.get(ib, xb, vb);
  const SpringAdj<R> t = spring_adjoint_terms<R>(a, xa, xb, va, vb, gvinc[ia], gvinc[ib], act, in.l0, in.k,
                                                 in.coef);
  if (in.side == 0) {
    gxs[0] += t.gd0; gxs[1] += t.gd1; gxs[2] += t.gd2;
    gvs[0] += t.h0; gvs[1] += t.h1; gvs[2] += t.h2;
    if (in.out >= 0) atomicAdd(gout + in.out, spring_gact<R>(t.gact, act, act_seed_scale, act_lim, act_seed));
  } else {
    gxs[0] -= t.gd0; gxs[1] -= t.gd1; gxs[2] -= t.gd2;
    gvs[0] -= t.h0; gvs[1] -= t.h1; gvs[2] -= t.h2;
  }
}

// The same with each spring's adjoint evaluated once: phase A (spring-
// parallel) stores gd and h per spring in adj[2 s], adj[2 s + 1] and adds the
// actuation gradient, phase B is spring_adjoint_gather's half-warp gather over
// the table (same lanes, same order).  For robots whose table fits in shared
// memory, in the fused reverse kernel (MsArgs::adj_cap).
template <typename R>
__device__ __forceinline__ void spring_adjoint_table(const MsArgs<R>& a, const RobotDesc& rb,
                                                     const PairRows<R>& xv, const V4<R>* gvinc, const R* outv,
                                                     R* gout, V4<R>* adj, const PairRows<R>& gs,
                                                     R act_seed_scale, R act_lim, bool act_seed) {
  const unsigned long long pol = policy_evict_last();
  for (int sp = threadIdx.x; sp < rb.n_s; sp += blockDim.x) {
    const int4 ab = ldg_i4_hint(a.spr_ab + rb.spr_off + sp, pol);
    const V4<R> f = ldg4_hint<R>(a.spr_p + rb.spr_off + sp, pol);
    const R act = ab.z >= 0 ? outv[ab.z] : R(0);
    V4<R> xa, va, xb, vb;
    xv.get(ab.x, xa, va);
    xv.get(ab.y, xb, vb);
    const SpringAdj<R> t = spring_adjoint_terms<R>(a, xa, xb, va, vb, gvinc[ab.x], gvinc[ab.y], act, f.x, f.y,
                                                   f.z);
    V4<R> g; g.x = t.gd0; g.y = t.gd1; g.z = t.gd2; g.w = 0;
    V4<R> h; h.x = t.h0; h.y = t.h1; h.z = t.h2; h.w = 0;
    adj[2 * sp] = g;
    adj[2 * sp + 1] = h;
    if (ab.z >= 0) atomicAdd(gout + ab.z, spring_gact<R>(t.gact, act, act_seed_scale, act_lim, act_seed));
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = (threadIdx.x >> 5), nw = (blockDim.x >> 5);
  const int l16 = lane & 15, half = lane >> 4;
  const int* ptr = a.inc_ptr + rb.ptr_off;
  const int N = rb.n_v, stride = nw * 2;
  for (int vb0 = wid * 2; vb0 < N; vb0 += stride) {
    const int v = vb0 + half;
    R gxs[3] = {0, 0, 0}, gvs[3] = {0, 0, 0};
    if (v < N) {
      const int beg = ptr[v], end = ptr[v + 1];
      for (int q = beg + l16; q < end; q += 16) {
        const int4 in = ldg_i4_hint(a.inc_i + rb.inc_off + q, pol);
        const V4<R> g = adj[2 * in.z], h = adj[2 * in.z + 1];
        if (in.y == 0) {
          gxs[0] += g.x; gxs[1] += g.y; gxs[2] += g.z;
          gvs[0] += h.x; gvs[1] += h.y; gvs[2] += h.z;
        } else {
          gxs[0] -= g.x; gxs[1] -= g.y; gxs[2] -= g.z;
          gvs[0] -= h.x; gvs[1] -= h.y; gvs[2] -= h.z;
        }
      }
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gxs[c] += __shfl_xor_sync(0xffffffffu, gxs[c], o);
        gvs[c] += __shfl_xor_sync(0xffffffffu, gvs[c], o);
      }
    }
    if (l16 == 0 && v < N) {
      V4<R> x, w;
      gs.get(v, x, w);
      x.x += gxs[0]; x.y += gxs[1]; x.z += gxs[2];
      w.x += gvs[0]; w.y += gvs[1]; w.z += gvs[2];
      gs.set(v, x, w);
    }
  }
}

// Each half-warp prefetches the first incidence record of U vertices before
// computing (as gather_vinc_all does), so U records per lane are in flight;
// every vertex's lanes, entries and shuffle tree are unchanged, so d x and
// d v are the same bits for any U.  Measured on the 512-robot uneven batch
// (151 substeps): reverse launches 31.9 / 31.0 / 31.9 / 41.9 ms for U = 1 /
// 2 / 4 / 8 (U = 8 spills).
#ifndef CLS_ADJ_U
#define CLS_ADJ_U 2
#endif
template <typename R>
__device__ __forceinline__ void spring_adjoint_gather(const MsArgs<R>& a, const RobotDesc& rb,
                                                      const PairRows<R>& xv, const V4<R>* gvinc, const R* outv,
                                                      R* gout, const PairRows<R>& gs, R act_seed_scale,
                                                      R act_lim, bool act_seed) {
  constexpr int U = CLS_ADJ_U;
  const unsigned long long pol = policy_evict_last();
  const int lane = threadIdx.x & 31, wid = (threadIdx.x >> 5), nw = (blockDim.x >> 5);
  const int l16 = lane & 15, half = lane >> 4;
  const int* ptr = a.inc_ptr + rb.ptr_off;
  const int N = rb.n_v, stride = nw * 2;
  // the loop bound is warp-uniform (vb0), so every shuffle below has all 32 lanes
  for (int vb0 = wid * 2; vb0 < N; vb0 += stride * U) {
    const int vb = vb0 + half;
    int beg[U], end[U];
    Inc<R> first[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int v = vb + k * stride;
      beg[k] = 0;
      end[k] = 0;
      if (v < N) { beg[k] = ptr[v]; end[k] = ptr[v + 1]; }
      const int q = beg[k] + l16;
      if (q < end[k]) first[k] = load_inc<R>(a, rb, q, pol);
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int v = vb + k * stride;
      R gxs[3] = {0, 0, 0}, gvs[3] = {0, 0, 0};
      if (v < N) {
        int q = beg[k] + l16;
        if (q < end[k])
          spring_adjoint_one<R>(a, first[k], v, xv, gvinc, outv, gout, act_seed_scale, act_lim, act_seed, gxs,
                                gvs);
        for (q += 16; q < end[k]; q += 16)
          spring_adjoint_one<R>(a, load_inc<R>(a, rb, q, pol), v, xv, gvinc, outv, gout, act_seed_scale,
                                act_lim, act_seed, gxs, gvs);
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          gxs[c] += __shfl_xor_sync(0xffffffffu, gxs[c], o);
          gvs[c] += __shfl_xor_sync(0xffffffffu, gvs[c], o);
        }
      }
      if (l16 == 0 && v < N) {
        V4<R> x, w;
        gs.get(v, x, w);
        x.x += gxs[0]; x.y += gxs[1]; x.z += gxs[2];
        w.x += gvs[0]; w.y += gvs[1]; w.z += gvs[2];
        gs.set(v, x, w);
      }
    }
  }
}

// ---------------------------------------------------------------- reverse
// The two halves of the adjoint of substep t around the controller, shared
// by the fused segment kernel and the batched-controller step kernels.

// Adjoint of substep t up to the controller outputs: x(t), v(t) from the
// records (slot kslot), advance_toi adjoint, spring-force adjoint, then
// dz of the output layer (recorded, and left in s.dz).
template <typename R>
__device__ __forceinline__ void rev_pre(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                        const RevSmem<R>& s, int e, int t, int kslot) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int N = rb.n_v, L = rb.n_layers;
  const R Br = R(rb.loss_envs);
  const R* bout = a.bias + rb.b_off[L - 1];
  const int nout = rb.n_out;
  const R* zl = a.rec_z + a.z_base[L - 1] + (size_t)kslot * a.z_total[L - 1] + ed.z_off[L - 1];
  {
    const V4<R>* rx = a.rec_x + (size_t)kslot * a.v_total + ed.v_off;
    const V4<R>* rv = a.rec_v + (size_t)kslot * a.v_total + ed.v_off;
    // with v_inc[t] as recorded by the forward pass (into gvinc as scratch)
    const V4<R>* rvi = a.rec_vinc + (size_t)kslot * a.v_total + ed.v_off;
    for (int i = tid; i < N; i += nt) { s.xv.set(i, rx[i], rv[i]); s.gvinc[i] = rvi[i]; }
    for (int o = tid; o < nout; o += nt) {
      s.bufA[o] = act_f<R>(a.act_out, zl[o] + bout[o]);
      s.bufB[o] = 0;
    }
  }
  __syncthreads();
  // adjoint of advance_toi(t + 1)
  for (int i = tid; i < N; i += nt) {
    V4<R> x, v, gx1, gv1;
    s.xv.get(i, x, v);
    s.g.get(i, gx1, gv1);
    const V4<R> vi = s.gvinc[i];
    R ov0 = a.drag_s * v.x + vi.x;
    R ov1 = a.drag_s * v.y + a.dt * a.gravity + vi.y;
    R ov2 = a.drag_s * v.z + vi.z;
    R nv0 = ov0, nv1 = ov1, nv2 = ov2, toi = 0, f = 0;
    const R nx1 = x.y + a.dt * ov1;
    const bool hit = (nx1 < a.ground && ov1 < R(-1e-4));
    if (hit) {
      toi = -(x.y - a.ground) / ov1;
      f = a.friction * (-ov1);
      nv1 = 0;
      nv0 = (ov0 < 0) ? fmin(R(0), ov0 + f) : fmax(R(0), ov0 - f);
      nv2 = (ov2 < 0) ? fmin(R(0), ov2 + f) : fmax(R(0), ov2 - f);
    }
    R gox0 = gx1.x, gox1 = gx1.y, gox2 = gx1.z;
    R gov0 = toi * gx1.x, gov1 = toi * gx1.y, gov2 = toi * gx1.z;
    const R dtt = a.dt - toi;
    const R gnv0 = dtt * gx1.x + gv1.x, gnv1 = dtt * gx1.y + gv1.y, gnv2 = dtt * gx1.z + gv1.z;
    const R gtoi = gx1.x * ov0 - gx1.x * nv0 + gx1.y * ov1 - gx1.y * nv1 + gx1.z * ov2 - gx1.z * nv2;
    if (hit) {
      R gf = 0;
      if (ov0 < 0) { if (!(R(0) < ov0 + f)) { gov0 += gnv0; gf += gnv0; } }
      else { if (!(ov0 - f < R(0))) { gov0 += gnv0; gf -= gnv0; } }
      if (ov2 < 0) { if (!(R(0) < ov2 + f)) { gov2 += gnv2; gf += gnv2; } }
      else { if (!(ov2 - f < R(0))) { gov2 += gnv2; gf -= gnv2; } }
      gov1 += -a.friction * gf;
      gox1 += -gtoi / ov1;
      gov1 += gtoi * (x.y - a.ground) / (ov1 * ov1);
    } else {
      gov0 += gnv0; gov1 += gnv1; gov2 += gnv2;
    }
    V4<R> gx0; gx0.x = gox0; gx0.y = gox1; gx0.z = gox2; gx0.w = 0;
    V4<R> gv0; gv0.x = a.drag_s * gov0; gv0.y = a.drag_s * gov1; gv0.z = a.drag_s * gov2; gv0.w = 0;
    V4<R> gvi; gvi.x = gov0; gvi.y = gov1; gvi.z = gov2; gvi.w = 0;
    s.g.set(i, gx0, gv0);
    s.gvinc[i] = gvi;
  }
  __syncthreads();
  // adjoint of apply_spring_force(t)
  {
    const size_t o = (size_t)t * a.n_envs + e;
    const int st_e = steps_of(a, e);
    const bool act_seed = (a.loss_mask & LOSS_ACTUATION) && t < st_e && a.th[o] < R(0.1 + 1e-4);
    const R lim = act_seed ? dpow_half<R>(dabs<R>(a.tv[o].x) / R(0.08)) : R(0);
    const R act_scale = R(10) / R(st_e) / Br / R(rb.n_s);
    if (s.adj)
      spring_adjoint_table<R>(a, rb, s.xv, s.gvinc, s.bufA, s.bufB, s.adj, s.g, act_scale, lim, act_seed);
    else
      spring_adjoint_gather<R>(a, rb, s.xv, s.gvinc, s.bufA, s.bufB, s.g, act_scale, lim, act_seed);
  }
  __syncthreads();
  // adjoint of the MLP's output activation
  {
    R* dzr = a.rec_dz + a.z_base[L - 1] + (size_t)kslot * a.z_total[L - 1] + ed.z_off[L - 1];
    for (int q = tid; q < nout; q += nt) {
      const R dz = s.bufB[q] * act_d<R>(a.act_out, zl[q] + bout[q]);
      s.dz[q] = dz;
      dzr[q] = dz;
    }
  }
  __syncthreads();
}

// Adjoint of substep t from the controller input on: s.bufA holds d loss /
// d (position columns of the input), s.xs holds x(t).  nn_input / center /
// loss seeds, then the running-height adjoint (hcarry carries d h across t).
template <typename R>
__device__ __forceinline__ void rev_post(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                         const RevSmem<R>& s, int e, int t, R& hcarry) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int N = rb.n_v;
  const R Br = R(rb.loss_envs);
  const R invN = R(1) / R(N);
  int* redi = reinterpret_cast<int*>(s.red + kRedInt);
  {
    const CenterVelocitySeed<R> vseed = load_center_velocity<R>(a, t, e, Br);
    R gc[3] = {0, 0, 0};
    for (int i = tid; i < N; i += nt) {
      const R g0 = s.bufA[3 * i] / R(0.2), g1 = s.bufA[3 * i + 1] / R(0.2), g2 = s.bufA[3 * i + 2] / R(0.2);
      R gxi[3] = {g0, g1, g2};
      gc[0] -= g0; gc[1] -= g1; gc[2] -= g2;
      if (a.x_full) seed_x_rotation_pose<R>(a, rb, ed, t, e, i, s.xv.p(i), Br, gxi, gc);
      s.g.add_p(i, gxi[0], gxi[1], gxi[2]);
    }
    block_sum<R, 3>(gc, s.red);
    apply_center_velocity<R>(vseed, gc);
    for (int i = tid; i < N; i += nt) s.g.add_p(i, gc[0] * invN, gc[1] * invN, gc[2] * invN);
  }
  // adjoint of compute_height (running max of the lowest point) and upper height
  if (a.loss_mask & (LOSS_HEIGHT | LOSS_CRAWL)) {
    const R gh = seed_height<R>(a, t, e, Br) + hcarry;
    const R gu = seed_upper<R>(a, t, e, Br);
    hcarry = 0;
    if (gh != R(0)) {
      R lo = R(10); int li = -1;
      for (int i = tid; i < N; i += nt) {
        const R y = s.xv.lo[i].y;
        if (!(lo < y)) { lo = y; li = i; }
      }
      block_argext<R>(lo, li, true, s.red, redi);
      R gmin = gh;
      if (t % a.jump_period != 0) {
        const R prev = a.obs_height[(size_t)(t - 1) * a.n_envs + e];
        if (lo < prev) { hcarry = gh; gmin = 0; }
      }
      if (tid == 0 && li >= 0 && gmin != R(0)) s.g.lo[li].y += gmin;
    }
    if (gu != R(0)) {
      R hi = R(-10); int hix = -1;
      for (int i = tid; i < N; i += nt) {
        const R y = s.xv.lo[i].y;
        if (!(y < hi)) { hi = y; hix = i; }
      }
      block_argext<R>(hi, hix, false, s.red, redi);
      if (tid == 0 && hix >= 0) s.g.lo[hix].y += gu;
    }
  }
  __syncthreads();
}

// Adjoint carry at the start of a reverse range: for the last segment the
// direct loss terms at x[t_end] (x[steps-1] is written by the last advance but
// never passed through pre_advance), else the carry left by the later segment.
template <typename R>
__device__ __forceinline__ void rev_load_carry(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                               const RevSmem<R>& s, int e, int t_end, bool last_seg,
                                               R& hcarry) {
  const int tid = threadIdx.x, nt = blockDim.x, N = rb.n_v;
  const R Br = R(rb.loss_envs);
  hcarry = 0;
  if (last_seg) {
    for (int i = tid; i < N; i += nt) {
      R gxi[3] = {0, 0, 0}, gcd[3] = {0, 0, 0};
      if (a.x_full) {
        const V4<R> xi = a.x_full[(size_t)t_end * a.v_total + ed.v_off + i];
        seed_x_rotation_pose<R>(a, rb, ed, t_end, e, i, xi, Br, gxi, gcd);
      }
      V4<R> g; g.x = gxi[0]; g.y = gxi[1]; g.z = gxi[2]; g.w = 0;
      V4<R> z; z.x = z.y = z.z = z.w = 0;
      s.g.set(i, g, z);
    }
  } else {
    for (int i = tid; i < N; i += nt) s.g.set(i, a.adj_x[ed.v_off + i], a.adj_v[ed.v_off + i]);
    hcarry = a.adj_h[e];
  }
  __syncthreads();
}

template <typename R>
__device__ __forceinline__ void rev_store_carry(const MsArgs<R>& a, const RobotDesc& rb, const EnvDesc& ed,
                                                const RevSmem<R>& s, int e, R hcarry) {
  const int tid = threadIdx.x, nt = blockDim.x, N = rb.n_v;
  for (int i = tid; i < N; i += nt) {
    V4<R> gx, gv;
    s.g.get(i, gx, gv);
    a.adj_x[ed.v_off + i] = gx;
    a.adj_v[ed.v_off + i] = gv;
  }
  if (tid == 0) a.adj_h[e] = hcarry;
  __syncthreads();
}

template <typename R, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
ms_reverse_kernel(MsArgs<R> a, int t_begin0, int t_end0, int last_seg0) {
  extern __shared__ __align__(256) char smem_raw[];
  __shared__ RobotDesc rb;
  __shared__ EnvDesc ed;
  __shared__ int s_item;
  RevSmem<R> s = carve_rev<R>(smem_raw, a);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (;;) {
    const int item = next_item(a, &s_item);
    if (item >= a.n_items) break;
    const int e = a.order[item];
    int t_begin = t_begin0, t_end = t_end0, last_seg = last_seg0;
    if (a.win) {
      const int4 w = a.win[e];
      t_begin = w.x; t_end = w.y; last_seg = w.w;
    }
    load_descs(a, e, rb, ed);
    const int N = rb.n_v, L = rb.n_layers;
    R hcarry = 0;
    if (s.w) load_controller_smem<R>(a.w, a.bias, rb, s.w, s.b);  // read after the syncs below
    rev_load_carry<R>(a, rb, ed, s, e, t_end, last_seg != 0, hcarry);
    __syncthreads();
    CLS_PHASE_START();
    for (int t = t_end - 1; t >= t_begin; --t) {
      const int kk = t - t_begin;
      rev_pre<R>(a, rb, ed, s, e, t, kk);
      CLS_PHASE(a, 3);
      // hidden layers of the MLP adjoint
      for (int l = L - 1; l >= 1; --l) {
        const int nin = rb.width[l];
        if (s.w)
          dense_transposed<R, true>(s.w + (rb.w_off[l] - rb.w_off[0]), rb.pitch[l], rb.width[l + 1], nin,
                                    s.dz, s.part, reinterpret_cast<V4<R>*>(s.bufA));
        else
          dense_transposed<R, false>(a.w + rb.w_off[l], rb.pitch[l], rb.width[l + 1], nin, s.dz, s.part,
                                     reinterpret_cast<V4<R>*>(s.bufA));
        const R* zp = a.rec_z + a.z_base[l - 1] + (size_t)kk * a.z_total[l - 1] + ed.z_off[l - 1];
        R* dzr = a.rec_dz + a.z_base[l - 1] + (size_t)kk * a.z_total[l - 1] + ed.z_off[l - 1];
        const R* bp = s.w ? s.b + (rb.b_off[l - 1] - rb.b_off[0]) : a.bias + rb.b_off[l - 1];
        for (int q = tid; q < nin; q += nt) {
          const R dz = s.bufA[q] * act_d<R>(a.act_hidden, zp[q] + bp[q]);
          s.dz[q] = dz;
          dzr[q] = dz;
        }
        __syncthreads();
      }
      // first layer: only the position columns carry state dependence
      if (s.w)
        dense_transposed<R, true>(s.w, rb.pitch[0], rb.width[1], 3 * N, s.dz, s.part,
                                  reinterpret_cast<V4<R>*>(s.bufA));
      else
        dense_transposed<R, false>(a.w + rb.w_off[0], rb.pitch[0], rb.width[1], 3 * N, s.dz, s.part,
                                   reinterpret_cast<V4<R>*>(s.bufA));
      CLS_PHASE(a, 6);
      rev_post<R>(a, rb, ed, s, e, t, hcarry);
      CLS_PHASE(a, 8);
    }
    rev_store_carry<R>(a, rb, ed, s, e, hcarry);
  }
}

// ------------------------------------------------------------------ losses
// Per-env loss terms (taichi_env.py:185-293) from the stored observables.
// out[e * 8 + slot]: raw sums (reference's loss_x, not multiplied by B);
// slot 7 holds the env's max height seen by the height loss.
template <typename R>
__global__ void ms_loss_kernel(MsArgs<R> a, double* out, const int* envs) {
  const int e = envs ? envs[blockIdx.x] : (int)blockIdx.x;  // envs: the listed envs only
  if (e >= a.n_envs) return;
  __shared__ double red[32 * 8];
  const EnvDesc ed = a.envs[e];
  const RobotDesc& rb = a.robots[ed.robot];
  const int N = rb.n_v, st = steps_of(a, e), rp = a.run_period, tp = a.turn_period, jp = a.jump_period;
  const double Br = rb.loss_envs;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  acc[7] = 0.0;
  const int tmax = (st < a.T - 1) ? st : a.T - 1;
  for (int t = threadIdx.x; t <= tmax; t += blockDim.x) {
    const size_t o = (size_t)t * a.n_envs + e;
    if ((a.loss_mask & LOSS_VELOCITY) && t >= rp && t % tp > rp) {
      const V4<R> c1 = a.obs_center[o], c0 = a.obs_center[o - (size_t)rp * a.n_envs];
      const V4<R> tv = a.tv[o - (size_t)rp * a.n_envs];
      const double ex = (double)c1.x - (double)c0.x - (double)tv.x;
      const double ez = (double)c1.z - (double)c0.z - (double)tv.z;
      acc[LS_VEL] += ex * ex / Br / st * 100 + ez * ez / Br / st * 100;
    }
    if ((a.loss_mask & LOSS_HEIGHT) && t >= 1 && t % jp == jp - 1 && (double)a.th[o] > 0.1 + 1e-6) {
      const double d = (double)a.obs_height[o] - (double)a.th[o];
      acc[LS_HEIGHT] += d * d / Br / (st / jp) * 100;
      acc[7] = fmax(acc[7], (double)a.obs_height[o]);
    }
    if ((a.loss_mask & LOSS_CRAWL) && t >= 1 && (double)a.tc[o] > 1 - 1e-4) {
      const double d = fmax((double)a.obs_upper[o] - 0.1, 0.0);
      acc[LS_CRAWL] += d * d / Br / st * 5.;
    }
    if ((a.loss_mask & LOSS_ACTUATION) && t < st && a.act_full && (double)a.th[o] < 0.1 + 1e-4) {
      const double lim = sqrt(fabs((double)a.tv[o].x) / 0.08);
      const R* af = a.act_full + (size_t)t * a.z_total[rb.n_layers - 1] + ed.z_off[rb.n_layers - 1];
      for (int s2 = 0; s2 < rb.n_s; ++s2) {
        const int q = a.spring_out[rb.spr_off + s2];
        const double act = q >= 0 ? (double)af[q] : 0.0;
        acc[LS_ACT] += fmax(fabs(act) - lim, 0.0) / rb.n_s / Br / st * 10;
      }
    }
  }
  // per-vertex terms over the trajectory: one warp per substep, its lanes
  // over the vertices (coalesced rows of x_full)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((a.loss_mask & (LOSS_ROTATION | LOSS_POSE)) && a.x_full) {
    for (int t = 1 + wid; t <= tmax; t += nw) {
      const size_t o = (size_t)t * a.n_envs + e;
      const V4<R>* xt = a.x_full + (size_t)t * a.v_total + ed.v_off;
      if ((a.loss_mask & LOSS_ROTATION) && t % tp > rp) {
        const V4<R> c1 = a.obs_center[o], c0 = a.obs_center[o - (size_t)rp * a.n_envs];
        const double ang = (double)a.th[o - (size_t)rp * a.n_envs] * 72. / 180. * 3.1415926535;
        const double ca = cos(ang), sn = sin(ang);
        const V4<R>* xr = a.x_full + (size_t)(t - rp) * a.v_total + ed.v_off;
        for (int i = lane; i < N; i += 32) {
          const V4<R> x1 = xt[i], x0 = xr[i];
          const double t0x = (double)x1.x - c1.x, t0y = (double)x1.y - c1.y, t0z = (double)x1.z - c1.z;
          const double t1x = (double)x0.x - c0.x, t1y = (double)x0.y - c0.y, t1z = (double)x0.z - c0.z;
          const double ex = t0x - (ca * t1x - sn * t1z), ey = t0y - t1y, ez = t0z - (sn * t1x + ca * t1z);
          acc[LS_ROT] += (ex * ex + ey * ey + ez * ez) / st / 40;
        }
      }
      if ((a.loss_mask & LOSS_POSE) && t % jp == 0) {
        for (int i = lane; i < N; i += 32) {
          const V4<R> x1 = xt[i];
          const V4<R> p = a.init_obj[ed.v_off + i];
          const double dx = (double)x1.x - p.x, dy = (double)x1.y - p.y, dz = (double)x1.z - p.z;
          acc[LS_POSE] += (dx * dx + dy * dy + dz * dz) / Br / (st / jp);
        }
      }
    }
  }
  // deterministic block reduction (max for slot 7)
  for (int m = 0; m < 8; ++m) {
    double v = acc[m];
    for (int off = 16; off > 0; off >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, off);
      v = (m == 7) ? fmax(v, w) : v + w;
    }
    if (lane == 0) red[m * 32 + wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    const int m = threadIdx.x;
    double v = red[m * 32];
    for (int w = 1; w < nw; ++w) v = (m == 7) ? fmax(v, red[m * 32 + w]) : v + red[m * 32 + w];
    out[(size_t)e * 8 + m] = v;
  }
}

// --------------------------------------------------- weight-gradient products
// dW_l[i, j] += sum over rows rho = (substep k of the segment, env of the type)
//   dz_l[rho, i] * a_l[rho, j]
// with a_0 the compact input record and a_l = act(z_{l-1} + b_{l-1}).  One CTA
// computes a 64 x 64 tile; 256 threads, 4 x 4 outputs each.
struct GemmTile {
  int robot, layer, i0, j0;
  int split, nsplit;  // split-K: this tile sums rows [rows*split/nsplit, rows*(split+1)/nsplit)
};

template <typename R>
__global__ void __launch_bounds__(256)
ms_wgrad_kernel(MsArgs<R> a, const GemmTile* tiles, int kseg, R* gw, R* gb) {
  constexpr int TM = 64, TN = 64, TK = 16;
  static_assert(TK * TM / 4 == 256 && TK * TN / 4 == 256, "one 4-value group per thread and operand");
  __shared__ __align__(32) R sA[TK][TM];
  __shared__ __align__(32) R sB[TK][TN];
  const GemmTile tl = tiles[blockIdx.x];
  const RobotDesc& rb = a.robots[tl.robot];
  const int l = tl.layer;
  const int M = rb.width[l + 1], Ncol = rb.width[l], pitch = rb.pitch[l];
  // per-env row strides of the records (rows padded to multiples of 4)
  const int zp = (M + 3) & ~3, ap = (Ncol + 3) & ~3;
  const int nb = rb.n_env;
  const EnvDesc& e0 = a.envs[rb.env_first];
  if (a.win) {  // served batches: one env per robot, its own window
    const int4 w = a.win[rb.env_first];
    kseg = w.y > w.x ? w.y - w.x : 0;
  }
  const int rows = kseg * nb;
  const int row_lo = (int)((long long)rows * tl.split / tl.nsplit);
  const int row_hi = (int)((long long)rows * (tl.split + 1) / tl.nsplit);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  R acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = 0;
  R bacc[4] = {0, 0, 0, 0};
  const R* biasp = (l > 0) ? a.bias + rb.b_off[l - 1] : nullptr;
  // staging: thread (rr, c4) loads 4 consecutive values of row rr of each
  // operand in one 16-byte access (record rows are padded to 4 values and
  // start on 4-value boundaries); padding columns of a row are read but
  // only reach outputs that are not stored
  const int rr = threadIdx.x >> 4, c4 = (threadIdx.x & 15) * 4;
  const int rin = l == 0 ? rb.pitch[0] : ap;  // B-operand row length in the records
  for (int r0 = row_lo; r0 < row_hi; r0 += TK) {
    {
      const int rho = r0 + rr;
      V4<R> va, vb;
      va.x = va.y = va.z = va.w = 0;
      vb = va;
      if (rho < row_hi) {
        const int k = rho / nb, b = rho - k * nb;
        const int i = tl.i0 + c4, j = tl.j0 + c4;
        if (i < zp)
          va = ldg4<R>(reinterpret_cast<const V4<R>*>(
              a.rec_dz + a.z_base[l] + (size_t)k * a.z_total[l] + e0.z_off[l] + (size_t)b * zp + i));
        if (j < rin) {
          if (l == 0) {
            vb = ldg4<R>(reinterpret_cast<const V4<R>*>(a.rec_in + (size_t)k * a.in_total + e0.in_off +
                                                        (size_t)b * rin + j));
          } else {
            const V4<R> z = ldg4<R>(reinterpret_cast<const V4<R>*>(
                a.rec_z + a.z_base[l - 1] + (size_t)k * a.z_total[l - 1] + e0.z_off[l - 1] + (size_t)b * ap + j));
            vb.x = j < Ncol ? act_f<R>(a.act_hidden, z.x + biasp[j]) : R(0);
            vb.y = j + 1 < Ncol ? act_f<R>(a.act_hidden, z.y + biasp[j + 1]) : R(0);
            vb.z = j + 2 < Ncol ? act_f<R>(a.act_hidden, z.z + biasp[j + 2]) : R(0);
            vb.w = j + 3 < Ncol ? act_f<R>(a.act_hidden, z.w + biasp[j + 3]) : R(0);
          }
        }
      }
      *reinterpret_cast<V4<R>*>(&sA[rr][c4]) = va;
      *reinterpret_cast<V4<R>*>(&sB[rr][c4]) = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      R av[4], bv[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) av[p] = sA[kk][ty * 4 + p];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = sB[kk][tx * 4 + q];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] += av[p] * bv[q];
        if (tl.j0 == 0 && tx == 0) bacc[p] += av[p];
      }
    }
    __syncthreads();
  }
  R* W = gw + rb.w_off[l];
  const bool split = tl.nsplit > 1;  // several CTAs add into this tile
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = tl.i0 + ty * 4 + p;
    if (i >= M) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = tl.j0 + tx * 4 + q;
      if (j < Ncol) {
        if (split) atomicAdd(W + (size_t)i * pitch + j, acc[p][q]);
        else W[(size_t)i * pitch + j] += acc[p][q];
      }
    }
    if (tl.j0 == 0 && tx == 0) {
      if (split) atomicAdd(gb + rb.b_off[l] + i, bacc[p]);
      else gb[rb.b_off[l] + i] += bacc[p];
    }
  }
}

// ------------------------------------------------- full <-> compact weights
// Column map of the first layer: the reference input
//   [n_sin sinusoids | per vertex (pos xyz, vel xyz = 0) | dup_v x (vx, vz) | dup_h x h | dup_c x c]
// (taichi_env.py:149-183) is stored compactly as
//   [pos (3N) | pad to 4 | n_sin sinusoids | vx, vz | h | c]
// velocity slots are always zero and duplicated goal columns always see equal
// inputs, so W_c[:, col] = sum of the reference columns that map to col.
__device__ __forceinline__ int full_to_compact(int j, int N, int pos_pad, int n_sin, int dup_v,
                                               int dup_h, int dup_c) {
  if (j < n_sin) return pos_pad + j;
  int q = j - n_sin;
  if (q < 6 * N) {
    const int v = q / 6, r = q - 6 * v;
    return r < 3 ? 3 * v + r : -1;
  }
  q -= 6 * N;
  int g = pos_pad + n_sin;
  if (q < 2 * dup_v) return g + (q & 1);
  q -= 2 * dup_v;
  if (dup_v > 0) g += 2;
  if (q < dup_h) return g;
  q -= dup_h;
  if (dup_h > 0) g += 1;
  if (q < dup_c) return g;
  return -1;
}

// Pack reference-layout master weights (float64 or R) into the compact layout.
template <typename R>
__global__ void ms_pack_weights_kernel(const R* __restrict__ master, long long m_off, int rows,
                                       int n_in_full, R* __restrict__ wc, long long c_off, int pitch,
                                       int layer, int N, int pos_pad, int n_sin, int dup_v, int dup_h,
                                       int dup_c) {
  const long long total = (long long)rows * pitch;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / pitch), c = (int)(q % pitch);
    const R* row = master + m_off + (long long)i * n_in_full;
    R s = 0;
    if (layer > 0) {
      s = c < n_in_full ? row[c] : R(0);
    } else if (c < 3 * N) {
      const int v = c / 3, d = c - 3 * v;
      s = row[n_sin + 6 * v + d];
    } else if (c >= pos_pad && c < pos_pad + n_sin) {
      s = row[c - pos_pad];
    } else if (c >= pos_pad + n_sin) {
      const int g = c - pos_pad - n_sin;
      const int base = n_sin + 6 * N;
      int gi = 0;
      if (dup_v > 0) {
        if (g < 2)
          for (int m = 0; m < dup_v; ++m) s += row[base + 2 * m + g];
        gi = 2;
      }
      if (dup_h > 0) {
        if (g == gi)
          for (int m = 0; m < dup_h; ++m) s += row[base + 2 * dup_v + m];
        gi += 1;
      }
      if (dup_c > 0 && g == gi)
        for (int m = 0; m < dup_c; ++m) s += row[base + 2 * dup_v + dup_h + m];
    }
    wc[c_off + q] = s;
  }
}

// grads of the reference layout from the compact layout (for export)
template <typename R>
__global__ void ms_unpack_grad_kernel(const R* __restrict__ gc, long long c_off, int pitch, int rows,
                                      int n_in_full, int layer, int N, int pos_pad, int n_sin,
                                      int dup_v, int dup_h, int dup_c, double* __restrict__ out) {
  const long long total = (long long)rows * n_in_full;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / n_in_full), j = (int)(q % n_in_full);
    int c = j;
    if (layer == 0) c = full_to_compact(j, N, pos_pad, n_sin, dup_v, dup_h, dup_c);
    out[q] = c >= 0 ? (double)gc[c_off + (long long)i * pitch + c] : 0.0;
  }
}

template <typename R>
__global__ void ms_convert_kernel(const double* __restrict__ in, R* __restrict__ out, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = (R)in[q];
}

template <typename R>
__global__ void ms_to_double_kernel(const R* __restrict__ in, double* __restrict__ out, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x)
    out[q] = (double)in[q];
}

// xyz triples (double) <-> V4 state
template <typename R>
__global__ void ms_xyz_to_v4_kernel(const double* __restrict__ in, V4<R>* __restrict__ out, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    V4<R> r;
    r.x = (R)in[3 * q]; r.y = (R)in[3 * q + 1]; r.z = (R)in[3 * q + 2]; r.w = 0;
    out[q] = r;
  }
}

template <typename R>
__global__ void ms_v4_to_xyz_kernel(const V4<R>* __restrict__ in, double* __restrict__ out, long long n) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const V4<R> r = in[q];
    out[3 * q] = r.x; out[3 * q + 1] = r.y; out[3 * q + 2] = r.z;
  }
}

// counter-based uniform in [0, 1): splitmix64 of (seed, stream, index)
__device__ __forceinline__ double u01(unsigned long long seed, unsigned long long stream,
                                      unsigned long long idx) {
  unsigned long long z = seed * 0x9E3779B97F4A7C15ULL + stream * 0xD1B54A32D192ED03ULL + idx;
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------ whole-model optimiser step
// Adam (Model.adam_update, nn.py:184-191) on the reference-layout master
// weights, with the gradient read from the compact layout, plus the squared
// gradient norm over the reference layout (Model.get_TNS, nn.py:173-182).
// One launch updates every weight and bias tensor of every robot type.  The
// tensors are laid end to end in a global element index; OptSeg describes one
// tensor.  Each CTA takes a contiguous chunk of that index, finds its first
// tensor by binary search and walks forward.
struct OptSeg {
  long long start;      // first global element index
  long long m_off;      // offset in the master / moment arrays (reference layout)
  long long c_off;      // offset in the compact gradient (weights) or gb (biases)
  int rows, cols, pitch, layer;   // layer < 0: bias vector
  int n_v, pos_pad;
};

__device__ __forceinline__ int find_seg(const OptSeg* segs, int n, long long q) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].start <= q) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <typename R>
__global__ void __launch_bounds__(256)
ms_adam_all_kernel(const OptSeg* __restrict__ segs, int n_segs, long long total, int chunk,
                   R* __restrict__ wm, R* __restrict__ wmm, R* __restrict__ wmv,
                   const R* __restrict__ gw, R* __restrict__ bias, R* __restrict__ bm,
                   R* __restrict__ bv, const R* __restrict__ gb, int n_sin, int dup_v, int dup_h,
                   int dup_c, double lr, double b1, double b2, int iter, const int* iter_dev,
                   int apply, double* tns) {
  __shared__ int s_seg;
  __shared__ double red[8];
  if (iter < 0) iter = *iter_dev;
  const double bc1 = 1.0 - pow(b1, (double)(iter + 1)), bc2 = 1.0 - pow(b2, (double)(iter + 1));
  const long long q0 = (long long)blockIdx.x * chunk;
  if (q0 >= total) return;
  if (threadIdx.x == 0) s_seg = find_seg(segs, n_segs, q0);
  __syncthreads();
  int sg = s_seg;
  double acc = 0;
  const long long q1 = q0 + chunk < total ? q0 + chunk : total;
  for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    while (sg + 1 < n_segs && segs[sg + 1].start <= q) ++sg;
    const OptSeg& o = segs[sg];
    const long long e = q - o.start;
    R g;
    R *w, *m, *v;
    if (o.layer < 0) {
      g = gb[o.c_off + e];
      w = bias + o.m_off + e; m = bm + o.m_off + e; v = bv + o.m_off + e;
    } else {
      const int i = (int)(e / o.cols), j = (int)(e % o.cols);
      int c = j;
      if (o.layer == 0) c = full_to_compact(j, o.n_v, o.pos_pad, n_sin, dup_v, dup_h, dup_c);
      g = c >= 0 ? gw[o.c_off + (long long)i * o.pitch + c] : R(0);
      w = wm + o.m_off + e; m = wmm + o.m_off + e; v = wmv + o.m_off + e;
    }
    acc += (double)g * (double)g;
    if (apply) {
      const R mm = R(b1) * *m + R(1 - b1) * g;
      const R vv = R(b2) * *v + R(1 - b2) * g * g;
      *m = mm;
      *v = vv;
      *w -= (R(lr) * (mm / R(bc1))) / (sqrt(vv / R(bc2)) + R(1e-8));
    }
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    if (tns) atomicAdd(tns, t);
  }
}

// Compact weights of every robot and layer from the reference-layout master
// (one launch; segments index the compact layout, rows x pitch each).
template <typename R>
__global__ void __launch_bounds__(256)
ms_pack_all_kernel(const OptSeg* __restrict__ segs, int n_segs, long long total, int chunk,
                   const R* __restrict__ master, R* __restrict__ wc, int n_sin, int dup_v,
                   int dup_h, int dup_c) {
  __shared__ int s_seg;
  const long long q0 = (long long)blockIdx.x * chunk;
  if (q0 >= total) return;
  if (threadIdx.x == 0) s_seg = find_seg(segs, n_segs, q0);
  __syncthreads();
  int sg = s_seg;
  const long long q1 = q0 + chunk < total ? q0 + chunk : total;
  for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    while (sg + 1 < n_segs && segs[sg + 1].start <= q) ++sg;
    const OptSeg& o = segs[sg];
    const long long e = q - o.start;
    const int i = (int)(e / o.pitch), c = (int)(e % o.pitch);
    const R* row = master + o.m_off + (long long)i * o.cols;
    R s = 0;
    const int N = o.n_v, pos_pad = o.pos_pad;
    if (o.layer > 0) {
      s = c < o.cols ? row[c] : R(0);
    } else if (c < 3 * N) {
      const int vtx = c / 3, d = c - 3 * vtx;
      s = row[n_sin + 6 * vtx + d];
    } else if (c >= pos_pad && c < pos_pad + n_sin) {
      s = row[c - pos_pad];
    } else if (c >= pos_pad + n_sin) {
      const int g = c - pos_pad - n_sin;
      const int base = n_sin + 6 * N;
      int gi = 0;
      if (dup_v > 0) {
        if (g < 2)
          for (int m = 0; m < dup_v; ++m) s += row[base + 2 * m + g];
        gi = 2;
      }
      if (dup_h > 0) {
        if (g == gi)
          for (int m = 0; m < dup_h; ++m) s += row[base + 2 * dup_v + m];
        gi += 1;
      }
      if (dup_c > 0 && g == gi)
        for (int m = 0; m < dup_c; ++m) s += row[base + 2 * dup_v + dup_h + m];
    }
    wc[o.c_off + e] = s;
  }
}

// ------------------------------------------------- initialisation kernels
// Model.weights_init (nn.py:59-67) for every weight tensor of every robot in
// one launch: W = (u * 2 - 1) * sqrt(6 / fan_in), u uniform from a counter-
// based stream keyed by (seed, tensor, element).  Bias segments are skipped
// (the reference leaves biases untouched).
template <typename R>
__global__ void __launch_bounds__(256)
ms_weights_init_all_kernel(const OptSeg* __restrict__ segs, int n_segs, long long total, int chunk,
                           R* __restrict__ master, unsigned long long seed) {
  __shared__ int s_seg;
  const long long q0 = (long long)blockIdx.x * chunk;
  if (q0 >= total) return;
  if (threadIdx.x == 0) s_seg = find_seg(segs, n_segs, q0);
  __syncthreads();
  int sg = s_seg;
  const long long q1 = q0 + chunk < total ? q0 + chunk : total;
  for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    while (sg + 1 < n_segs && segs[sg + 1].start <= q) ++sg;
    const OptSeg& o = segs[sg];
    if (o.layer < 0) continue;
    const long long e = q - o.start;
    const double scale = sqrt(6.0 / o.cols);
    master[o.m_off + e] = (R)((u01(seed, (unsigned long long)sg, (unsigned long long)e) * 2 - 1) * scale);
  }
}

// TaichiEnv.initialize_train, 3D branch (taichi_env.py:385-447): one pool of
// three uniforms per (turn period, env); 25 % turn -1, 25 % turn +1, 25 %
// forward/backward along z, 25 % along x.  target_c is left unchanged.
template <typename R>
__global__ void ms_initialize_train_kernel(V4<R>* __restrict__ tv, R* __restrict__ th, int T,
                                           int steps, int n_envs, int turn_period,
                                           unsigned long long seed, int iter, double max_velocity) {
  const long long total = (long long)T * n_envs;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(q / n_envs), k = (int)(q % n_envs);
    if (t >= steps) continue;
    const unsigned long long base = ((unsigned long long)(t / turn_period) * n_envs + k) * 3;
    const double p0 = u01(seed, 0x7000000ULL + (unsigned long long)iter, base);
    const double p1 = u01(seed, 0x7000000ULL + (unsigned long long)iter, base + 1);
    V4<R> v; v.x = 0; v.y = 0; v.z = 0; v.w = 0;
    R h = 0;
    if (p0 < 0.25) {
      h = R(-1);
    } else if (p0 < 0.5) {
      h = R(1);
    } else if (p0 < 0.75) {
      v.z = (R)((p1 * 2. - 1.) * max_velocity);
    } else {
      v.x = (R)((p1 * 2. - 1.) * max_velocity);
    }
    tv[q] = v;
    th[q] = h;
  }
}

}  // namespace cls
