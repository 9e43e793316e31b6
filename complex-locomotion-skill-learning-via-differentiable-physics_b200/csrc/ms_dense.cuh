// ms_dense.cuh -- batched-controller path for robot types shared by many envs.
//
// The fused segment kernels run the controller MLP as one GEMV per env per
// substep, so every env streams the whole weight set each substep.  When
// hundreds to thousands of envs share one robot type (one controller), the
// controller of a substep is a dense contraction over the envs instead:
//   Z_l[env][o] = sum_i A_l[env][i] W_l[o][i],   A_0 = input row,
//   A_l = act(Z_{l-1} + b_{l-1}),
// and its adjoint G_l[env][i] = sum_o dZ_l[env][o] W_l[o][i].  Here a substep
// is split at the controller into launches:
//   forward:  step kernel (advance of t-1 with the outputs of t-1, then the
//             observables and input row of t) -> one GEMM per layer
//   reverse:  step kernel (input / centre / loss-seed adjoint of t+1, then the
//             advance and spring adjoints of t up to dZ of the output layer)
//             -> one GEMM per layer down to the position columns of the input
// The step kernels reuse the fused kernels' substep halves (fwd_pre/fwd_post,
// rev_pre/rev_post) with one CTA per env and the state in global memory
// between launches; the GEMMs run on the tensor cores (tcgen05, 3xTF32, FP32
// accumulate) for FP32 and as SIMT tiles for FP64.  Records use the fused
// path's layout (rows padded to 4 floats), so the weight-gradient kernel and
// the checkpoint schedule are shared.
#pragma once
#include <type_traits>

#include "ms_segment.cuh"
#include "umma_gemm.cuh"

namespace cls {


__host__ __device__ __forceinline__ int pad4(int x) { return (x + 3) & ~3; }

// ------------------------------------------------------------ step kernels
// One CTA per env; the substep halves with the env's state in the CTA's
// shared memory (the fused kernels' carve with the controller buffers sized
// for the output layer only).  One warp per env
// (several envs per CTA, no CTA barrier) measured slower.

// Forward step t of a range [t_first, t_end):
//   t > t_first: controller outputs of t-1 from the output layer's record
//                (slot k_prev), then spring forces and advance of t-1;
//   t < t_end:   checkpoint / records / observables of x(t), the input row of
//                t into record slot k_cur (zero padded) and, FP32, into the
//                first GEMM's pre-split operand; state to live_x/v;
//   t == t_end:  the range's end (checkpoint, final state).
// The state comes from checkpoint slot src_slot at t == t_first, else from
// live_x/v.
template <typename R, int MAXT>
__global__ void __launch_bounds__(MAXT)
ms_step_fwd_kernel(MsArgs<R> a, int t, int t_first, int t_end, int mode, int src_slot, int k_prev,
                   int k_cur) {
  extern __shared__ __align__(256) char smem_raw[];
  __shared__ RobotDesc rb;
  __shared__ EnvDesc ed;
  const int item = blockIdx.x;
  if (item >= a.n_items) return;
  FwdSmem<R> s = carve_fwd<R>(smem_raw, a);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int e = a.order[item];
  load_descs<R>(a, e, rb, ed);
  const int N = rb.n_v, L = rb.n_layers;
  CLS_PHASE_START();
  {
    const bool first = (t == t_first);
    const V4<R>* cx = first ? a.ckpt_x + (size_t)src_slot * a.v_total + ed.v_off : a.live_x + ed.v_off;
    const V4<R>* cv = first ? a.ckpt_v + (size_t)src_slot * a.v_total + ed.v_off : a.live_v + ed.v_off;
    for (int i = tid; i < N; i += nt) { s.xs[i] = cx[i]; s.vs[i] = cv[i]; }
  }
  __syncthreads();
  if (t > t_first) {
    const R* zl = a.rec_z + a.z_base[L - 1] + (size_t)k_prev * a.z_total[L - 1] + ed.z_off[L - 1];
    const R* bo = a.bias + rb.b_off[L - 1];
    for (int o = tid; o < rb.n_out; o += nt) s.buf0[o] = act_f<R>(a.act_out, zl[o] + bo[o]);
    __syncthreads();
    CLS_PHASE(a, 20);
    fwd_post<R>(a, rb, ed, s, t - 1, mode, k_prev, s.buf0);
    CLS_PHASE(a, 21);
  }
  if (t < t_end) {
    R hprev = 0;
    if ((mode & FWD_OBS) && t > 0) hprev = a.obs_height[(size_t)(t - 1) * a.n_envs + e];
    load_head_smem<R>(a, rb, ed, s, t, mode);
    fwd_pre<R>(a, rb, ed, s, e, t, t_first, mode, k_cur, true, true, hprev);
    CLS_PHASE(a, 22);
    if constexpr (std::is_same<R, float>::value) {
      // the input row as the first layer's pre-split A operand
      const umma::SplitTiles st{a.tiles + a.dense[ed.robot].ta_f[0], umma::TM, (rb.n_c + 31) / 32};
      const int j = e - rb.env_first;
      for (int q = 4 * tid; q < rb.n_c; q += 4 * nt)
        st.store4(j, q, make_float4(s.ain[q], s.ain[q + 1], s.ain[q + 2], s.ain[q + 3]));
    }
    CLS_PHASE(a, 23);
    for (int i = tid; i < N; i += nt) {
      a.live_x[ed.v_off + i] = s.xs[i];
      a.live_v[ed.v_off + i] = s.vs[i];
    }
    CLS_PHASE(a, 24);
  } else {
    fwd_finish<R>(a, rb, ed, s, t_first, t_end, mode);
  }
}

// Reverse step over a segment [t_begin, t_end):
//   t_post >= 0: adjoint of substep t_post from its controller input on
//                (d input positions in din, x(t_post) from the records);
//   t_pre >= 0:  adjoint of substep t_pre up to dZ of the output layer (and,
//                FP32, dZ as the adjoint GEMM's pre-split operand).
// The adjoint state is carried in adj_x/v/h between launches; the first
// launch of the segment (t_pre = t_end - 1) seeds it (last segment) or takes
// the carry of the later segment.
template <typename R, int MAXT>
__global__ void __launch_bounds__(MAXT)
ms_step_rev_kernel(MsArgs<R> a, int t_post, int t_pre, int t_begin, int t_end, int last_seg) {
  extern __shared__ __align__(256) char smem_raw[];
  __shared__ RobotDesc rb;
  __shared__ EnvDesc ed;
  const int item = blockIdx.x;
  if (item >= a.n_items) return;
  RevSmem<R> s = carve_rev<R>(smem_raw, a);
  const int tid = threadIdx.x, nt = blockDim.x;
  const int e = a.order[item];
  load_descs<R>(a, e, rb, ed);
  const int N = rb.n_v;
  R hcarry = 0;
  CLS_PHASE_START();
  rev_load_carry<R>(a, rb, ed, s, e, t_end, t_pre == t_end - 1 && last_seg != 0, hcarry);
  CLS_PHASE(a, 25);
  if (t_post >= 0) {
    const int kk = t_post - t_begin;
    const V4<R>* rx = a.rec_x + (size_t)kk * a.v_total + ed.v_off;
    for (int i = tid; i < N; i += nt) s.xv.lo[i] = rx[i];  // x(t_post) only: rev_post reads p
    const R* dp = a.din + (size_t)3 * ed.v_off;
    for (int q = tid; q < 3 * N; q += nt) s.bufA[q] = dp[q];
    __syncthreads();
    rev_post<R>(a, rb, ed, s, e, t_post, hcarry);
    CLS_PHASE(a, 26);
  }
  if (t_pre >= 0) {
    rev_pre<R>(a, rb, ed, s, e, t_pre, t_pre - t_begin);
    CLS_PHASE(a, 27);
    if constexpr (std::is_same<R, float>::value) {
      // dZ of the output layer as the adjoint GEMM's pre-split A operand
      const int no = rb.n_out;
      const umma::SplitTiles st{a.tiles + a.dense[ed.robot].ta_b[rb.n_layers - 1], umma::TM, (no + 31) / 32};
      const int j = e - rb.env_first;
      for (int q = 4 * tid; q < no; q += 4 * nt) {
        const float4 v = make_float4(s.dz[q], q + 1 < no ? s.dz[q + 1] : 0.f, q + 2 < no ? s.dz[q + 2] : 0.f,
                                     q + 3 < no ? s.dz[q + 3] : 0.f);
        st.store4(j, q, v);
      }
    }
    CLS_PHASE(a, 28);
  }
  rev_store_carry<R>(a, rb, ed, s, e, hcarry);
  CLS_PHASE(a, 29);
}

// ------------------------------------------------------------ GEMM operands
// Row pointers and element maps of one job, shared by the tensor-core and the
// SIMT tiles.  Forward (layer l): A = input rows (l = 0) or act(Z_{l-1} + b)
// (l > 0), B = W_l rows, C -> Z_l record.  Backward (layer l): A = dZ_l
// record rows, B = rows of W_l^T, C -> dZ_{l-1} = C * act'(Z_{l-1} + b) (l > 0)
// or d input positions (l = 0).
template <typename R>
struct FwdOperands {
  int act;         // hidden activation
  const R* arow;   // A row of env m0
  int astride, kin;
  const R* bprev;  // bias of layer l - 1 (l > 0) or null
  const R* W;      // row n0 of W_l
  int wpitch;
  R* zout;         // Z_l record, row m0, column n0
  int zstride;
  __device__ V4<R> load_a(int k, int i) const {
    V4<R> v = *reinterpret_cast<const V4<R>*>(arow + (size_t)i * astride + k);
    if (bprev) {
      const V4<R> b = *reinterpret_cast<const V4<R>*>(bprev + k);
      v.x = act_f<R>(act, v.x + b.x);
      v.y = act_f<R>(act, v.y + b.y);
      v.z = act_f<R>(act, v.z + b.z);
      v.w = act_f<R>(act, v.w + b.w);
    }
    if (k + 4 > kin) {  // padding columns
      if (k >= kin) v.x = 0;
      if (k + 1 >= kin) v.y = 0;
      if (k + 2 >= kin) v.z = 0;
      v.w = 0;
    }
    return v;
  }
  __device__ V4<R> load_b(int k, int j) const {
    return *reinterpret_cast<const V4<R>*>(W + (size_t)j * wpitch + k);
  }
  __device__ void store(int i, int j, R v) const { zout[(size_t)i * zstride + j] = v; }
};

template <typename R>
__device__ __forceinline__ FwdOperands<R> fwd_operands(const MsArgs<R>& a, const DenseJob& jb, int kslot,
                                                       int& m_valid, int& n_valid, int& kpad, int tm,
                                                       int tn) {
  const RobotDesc& rb = a.robots[jb.robot];
  const EnvDesc& e0 = a.envs[rb.env_first];
  const int l = jb.layer;
  FwdOperands<R> op;
  op.act = a.act_hidden;
  op.kin = rb.width[l];
  kpad = pad4(op.kin);
  if (l == 0) {
    op.astride = rb.pitch[0];
    op.arow = a.rec_in + (size_t)kslot * a.in_total + e0.in_off + (size_t)jb.m0 * op.astride;
    op.bprev = nullptr;
  } else {
    op.astride = kpad;
    op.arow = a.rec_z + a.z_base[l - 1] + (size_t)kslot * a.z_total[l - 1] + e0.z_off[l - 1] +
              (size_t)jb.m0 * op.astride;
    op.bprev = a.bias + rb.b_off[l - 1];
  }
  op.wpitch = rb.pitch[l];
  op.W = a.w + rb.w_off[l] + (size_t)jb.n0 * op.wpitch;
  op.zstride = pad4(rb.width[l + 1]);
  op.zout = a.rec_z + a.z_base[l] + (size_t)kslot * a.z_total[l] + e0.z_off[l] + (size_t)jb.m0 * op.zstride +
            jb.n0;
  m_valid = min(tm, rb.n_env - jb.m0);
  n_valid = min(tn, rb.width[l + 1] - jb.n0);
  return op;
}

template <typename R>
struct BwdOperands {
  int act;         // hidden activation
  const R* arow;   // dZ_l row of env m0
  int astride, kin;
  const R* WT;     // row n0 of W_l^T
  int wtpitch;
  // l > 0: dZ_{l-1} record (row m0, column n0), Z_{l-1} record, bias of l - 1
  R* dzout; const R* zin; const R* bprev; int ostride;
  // l = 0: d input positions (row m0, column n0), stride 3 n_v
  R* dinout;
  __device__ V4<R> load_a(int k, int i) const {
    V4<R> v = *reinterpret_cast<const V4<R>*>(arow + (size_t)i * astride + k);
    if (k + 4 > kin) {  // padding columns
      if (k >= kin) v.x = 0;
      if (k + 1 >= kin) v.y = 0;
      if (k + 2 >= kin) v.z = 0;
      v.w = 0;
    }
    return v;
  }
  __device__ V4<R> load_b(int k, int j) const {
    return *reinterpret_cast<const V4<R>*>(WT + (size_t)j * wtpitch + k);
  }
  __device__ void store(int i, int j, R v) const {
    if (dinout) {
      dinout[(size_t)i * ostride + j] = v;
    } else {
      const size_t o = (size_t)i * ostride + j;
      dzout[o] = v * act_d<R>(act, zin[o] + bprev[j]);
    }
  }
};

template <typename R>
__device__ __forceinline__ BwdOperands<R> bwd_operands(const MsArgs<R>& a, const DenseJob& jb, int kslot,
                                                       int& m_valid, int& n_valid, int& kpad, int tm,
                                                       int tn) {
  const RobotDesc& rb = a.robots[jb.robot];
  const EnvDesc& e0 = a.envs[rb.env_first];
  const int l = jb.layer;
  BwdOperands<R> op;
  op.act = a.act_hidden;
  op.kin = rb.width[l + 1];
  kpad = pad4(op.kin);
  op.astride = kpad;
  op.arow = a.rec_dz + a.z_base[l] + (size_t)kslot * a.z_total[l] + e0.z_off[l] + (size_t)jb.m0 * kpad;
  op.wtpitch = a.dense[jb.robot].wt_pitch[l];
  op.WT = a.wt + a.dense[jb.robot].wt_off[l] + (size_t)jb.n0 * op.wtpitch;
  int ncol;
  if (l > 0) {
    ncol = rb.width[l];
    op.ostride = pad4(ncol);
    const size_t base = a.z_base[l - 1] + (size_t)kslot * a.z_total[l - 1] + e0.z_off[l - 1] +
                        (size_t)jb.m0 * op.ostride + jb.n0;
    op.dzout = a.rec_dz + base;
    op.zin = a.rec_z + base;
    op.bprev = a.bias + rb.b_off[l - 1] + jb.n0;
    op.dinout = nullptr;
  } else {
    ncol = 3 * rb.n_v;
    op.ostride = ncol;
    op.dinout = a.din + (size_t)3 * (e0.v_off + (size_t)jb.m0 * rb.n_v) + jb.n0;
    op.dzout = nullptr; op.zin = nullptr; op.bprev = nullptr;
  }
  m_valid = min(tm, rb.n_env - jb.m0);
  n_valid = min(tn, ncol - jb.n0);
  return op;
}

// ------------------------------------------------------- tensor-core GEMMs
// FP32: one 128-env x 64-output tile per CTA, operands streamed as pre-split
// tiles (umma::tile_gemm_bulk).  The epilogue writes, along rows (16 bytes per
// thread), the FP32 record the adjoint and the weight-gradient products read
// and the next GEMM's pre-split A operand:
//   forward l:  Z_l record; act(Z_l + b_l) as layer l + 1's A (hidden layers)
//   adjoint l:  dZ_{l-1} = C act'(Z_{l-1} + b_{l-1}) record and as layer l-1's
//               adjoint A (l > 0); d input positions (l = 0)
#ifndef CLS_DENSE_TN
#define CLS_DENSE_TN 64
#endif
#ifndef CLS_BULK_STAGES
#define CLS_BULK_STAGES 4
#endif
constexpr int kDenseTN = CLS_DENSE_TN;        // output columns per tensor-core tile
constexpr int kBulkStages = CLS_BULK_STAGES;  // stages of the bulk-copy ring (4 x 48 KB at TN = 64)

__device__ __forceinline__ float4 mask4(float4 v, int col, int n) {
  if (col + 1 > n) v.x = 0.f;
  if (col + 2 > n) v.y = 0.f;
  if (col + 3 > n) v.z = 0.f;
  if (col + 4 > n) v.w = 0.f;
  return v;
}

template <int BWD>
__global__ void __launch_bounds__(umma::kBulkThreads)
ms_ctrl_gemm_tc_kernel(MsArgs<float> a, const DenseJob* jobs, int kslot) {
  extern __shared__ __align__(1024) float smem_f[];
  __shared__ umma::BulkShared bs;
  const DenseJob jb = jobs[blockIdx.x];
  const RobotDesc& rb = a.robots[jb.robot];
  const DenseDesc& dd = a.dense[jb.robot];
  const EnvDesc& e0 = a.envs[rb.env_first];
  const int l = jb.layer;
  const int kin = BWD ? rb.width[l + 1] : rb.width[l];
  const int nkt = (kin + 31) / 32;
  const float* ab = a.tiles + (BWD ? dd.ta_b[l] : dd.ta_f[l]) + (size_t)(jb.m0 / umma::TM) * nkt * 64 * umma::TM;
  const float* bb = a.tiles + (BWD ? dd.tb_b[l] : dd.tb_f[l]) + (size_t)(jb.n0 / kDenseTN) * nkt * 64 * kDenseTN;
  const int m_valid = min(umma::TM, rb.n_env - jb.m0);
  const int ncol = BWD ? (l > 0 ? rb.width[l] : 3 * rb.n_v) : rb.width[l + 1];
  const int n_valid = min(kDenseTN, ncol - jb.n0);
  const int act = a.act_hidden;
  const bool ok = umma::tile_gemm_bulk<kDenseTN, kBulkStages>(smem_f, bs, ab, bb, nkt, [&](const float* cs, int ld) {
    constexpr int C4 = kDenseTN / 4;
    for (int q = threadIdx.x; q < umma::TM * C4; q += blockDim.x) {
      const int i = q / C4, j = 4 * (q % C4);
      if (i >= m_valid || j >= n_valid) continue;
      const float4 v = *reinterpret_cast<const float4*>(cs + i * ld + j);
      const int row = jb.m0 + i, col = jb.n0 + j;
      if (!BWD) {
        const int w = rb.width[l + 1];
        float* zr = a.rec_z + a.z_base[l] + (size_t)kslot * a.z_total[l] + e0.z_off[l] + (size_t)row * pad4(w) + col;
        *reinterpret_cast<float4*>(zr) = v;
        if (l + 1 < rb.n_layers) {
          const float4 b = *reinterpret_cast<const float4*>(a.bias + rb.b_off[l] + col);
          const float4 y = make_float4(act_f<float>(act, v.x + b.x), act_f<float>(act, v.y + b.y),
                                       act_f<float>(act, v.z + b.z), act_f<float>(act, v.w + b.w));
          const umma::SplitTiles st{a.tiles + dd.ta_f[l + 1], umma::TM, (w + 31) / 32};
          st.store4(row, col, mask4(y, col, w));
        }
      } else if (l > 0) {
        const int w = rb.width[l];
        const size_t o = a.z_base[l - 1] + (size_t)kslot * a.z_total[l - 1] + e0.z_off[l - 1] + (size_t)row * pad4(w) + col;
        const float4 z = *reinterpret_cast<const float4*>(a.rec_z + o);
        const float4 b = *reinterpret_cast<const float4*>(a.bias + rb.b_off[l - 1] + col);
        const float4 dz = mask4(make_float4(v.x * act_d<float>(act, z.x + b.x), v.y * act_d<float>(act, z.y + b.y),
                                            v.z * act_d<float>(act, z.z + b.z), v.w * act_d<float>(act, z.w + b.w)),
                                col, w);
        *reinterpret_cast<float4*>(a.rec_dz + o) = dz;
        const umma::SplitTiles st{a.tiles + dd.ta_b[l - 1], umma::TM, (w + 31) / 32};
        st.store4(row, col, dz);
      } else {
        float* dp = a.din + (size_t)3 * (e0.v_off + (size_t)row * rb.n_v) + col;
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (j + u < n_valid) dp[u] = vv[u];
      }
    }
  }, umma::WaitPolicy{a.gemm_wait_limit, a.gemm_starve});
  if (!ok && threadIdx.x == 0) atomicOr(a.status, ERR_TIMEOUT);
  if (threadIdx.x < 32) umma::tmem_relinquish();
}


// --------------------------------------------- weight-gradient products (FP32)
// dW_l[o][i] = sum over the segment's (slot, env) rows of dZ_l[o] A_l[i] and
// db_l[o] = sum dZ_l[o]: a contraction over ~K x envs rows, run as the bulk
// tensor-core tile with M = outputs, N = inputs + 1 (a row of ones turns the
// bias gradient into the last column) and K = the rows.  First the FP32
// records are transposed into pre-split K-major tiles: one CTA moves 32 envs
// x 32 columns of kWgSlots record slots through shared memory, reading env
// rows (128 bytes each) and writing each column's 32 K values as one 128-byte
// line per precision part.
constexpr int kWgSlots = 10;  // record slots per transpose CTA

__global__ void __launch_bounds__(256)
ms_wgrad_transpose_kernel(MsArgs<float> a, const WgTrans* jobs, const WgCol* cols, int slot0, int nslots) {
  __shared__ float tile[32][33];
  const WgCol wc = cols[blockIdx.y];
  const WgTrans jb = jobs[wc.job];
  const RobotDesc& rb = a.robots[jb.robot];
  const DenseDesc& dd = a.dense[jb.robot];
  const EnvDesc& e0 = a.envs[rb.env_first];
  const int j0 = blockIdx.x * 32;
  if (j0 >= dd.nep) return;
  const int l = jb.layer, tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int rows = jb.cols + (jb.kind == 2 ? 0 : 1);
  const float* src0;
  int stride, slot;
  if (jb.kind == 0) {
    stride = rb.pitch[0];
    slot = a.in_total;
    src0 = a.rec_in + e0.in_off;
  } else if (jb.kind == 1) {
    stride = pad4(rb.width[l]);
    slot = a.z_total[l - 1];
    src0 = a.rec_z + a.z_base[l - 1] + e0.z_off[l - 1];
  } else {
    stride = pad4(rb.width[l + 1]);
    slot = a.z_total[l];
    src0 = a.rec_dz + a.z_base[l] + e0.z_off[l];
  }
  const float* bias = jb.kind == 1 ? a.bias + rb.b_off[l - 1] : nullptr;
  float* dst = a.wtiles + (jb.kind == 2 ? dd.tw_d[l] : dd.tw_a[l]);
  const int c = wc.c0 + tx;
  const float b = (bias && c < jb.cols) ? bias[c] : 0.f;
  const int kk1 = min(nslots, (int)(blockIdx.z + 1) * kWgSlots);
  for (int kk = blockIdx.z * kWgSlots; kk < kk1; ++kk) {
    const float* src = src0 + (size_t)(slot0 + kk) * slot;
    for (int r = ty; r < 32; r += 8) {
      const int j = j0 + r;
      float v = 0.f;
      if (j < rb.n_env) {
        if (c < jb.cols) {
          v = src[(size_t)j * stride + c];
          if (bias) v = act_f<float>(a.act_hidden, v + b);
        } else if (c == jb.cols && jb.kind != 2) {
          v = 1.f;
        }
      }
      tile[r][tx] = v;
    }
    __syncthreads();
    const int k = kk * dd.nep + j0 + tx;
    for (int r = ty; r < 32; r += 8) {
      const int cc = wc.c0 + r;
      if (cc >= rows) continue;
      // the tile height is a compile-time constant per operand (shifts, not divisions)
      if (jb.kind == 2) umma::SplitTiles{dst, umma::TM, dd.nkt_w}.store_tr<umma::TM>(cc, k, tile[tx][r]);
      else umma::SplitTiles{dst, kDenseTN, dd.nkt_w}.store_tr<kDenseTN>(cc, k, tile[tx][r]);
    }
    __syncthreads();
  }
}

// one 128-output x 64-input tile of one layer's weight gradient over K split
// `split` of the segment's nslots x nep rows; atomic adds (several splits
// and segments add into one gradient)
__global__ void __launch_bounds__(umma::kBulkThreads)
ms_wgrad_tc_kernel(MsArgs<float> a, const WgJob* jobs, int nslots, float* gw, float* gb) {
  extern __shared__ __align__(1024) float smem_f[];
  __shared__ umma::BulkShared bs;
  const WgJob jb = jobs[blockIdx.x];
  const RobotDesc& rb = a.robots[jb.robot];
  const DenseDesc& dd = a.dense[jb.robot];
  const int l = jb.layer;
  const int total = nslots * dd.nep / 32;
  const int k0 = (int)((long long)total * jb.split / jb.nsplit);
  const int k1 = (int)((long long)total * (jb.split + 1) / jb.nsplit);
  const float* ab = a.wtiles + dd.tw_d[l] + ((size_t)(jb.o0 / umma::TM) * dd.nkt_w + k0) * (64 * umma::TM);
  const float* bb = a.wtiles + dd.tw_a[l] + ((size_t)(jb.i0 / kDenseTN) * dd.nkt_w + k0) * (64 * kDenseTN);
  const int nout = rb.width[l + 1], nin = rb.width[l], pitch = rb.pitch[l];
  float* W = gw + rb.w_off[l];
  float* B = gb + rb.b_off[l];
  const bool ok = umma::tile_gemm_bulk<kDenseTN, kBulkStages>(
      smem_f, bs, ab, bb, k1 - k0, [&](const float* cs, int ld) {
        for (int q = threadIdx.x; q < umma::TM * kDenseTN; q += blockDim.x) {
          const int i = q / kDenseTN, j = q % kDenseTN;
          const int o = jb.o0 + i, c = jb.i0 + j;
          if (o >= nout || c > nin) continue;
          const float v = cs[i * ld + j];
          if (c < nin) atomicAdd(W + (size_t)o * pitch + c, v);
          else atomicAdd(B + o, v);
        }
      }, umma::WaitPolicy{a.gemm_wait_limit, a.gemm_starve});
  if (!ok && threadIdx.x == 0) atomicOr(a.status, ERR_TIMEOUT);
  if (threadIdx.x < 32) umma::tmem_relinquish();
}

// pre-split tiles of every layer's W_l (forward B: rows = outputs) and W_l^T
// (adjoint B: rows = inputs), one thread per weight
__global__ void __launch_bounds__(256) ms_split_weights_kernel(const float* __restrict__ w, float* tiles,
                                                               const SplitSeg* segs, int n_segs, long long total) {
  for (long long q = blockIdx.x * 256ll + threadIdx.x; q < total; q += (long long)gridDim.x * 256) {
    int lo = 0, hi = n_segs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (segs[mid].first <= q) lo = mid; else hi = mid - 1;
    }
    const SplitSeg sg = segs[lo];
    const long long r = q - sg.first;
    const int o = (int)(r / sg.cols), i = (int)(r % sg.cols);
    const float v = w[sg.w_off + (size_t)o * sg.pitch + i];
    umma::SplitTiles{tiles + sg.tf_off, kDenseTN, (sg.cols + 31) / 32}.store(o, i, v);
    umma::SplitTiles{tiles + sg.tb_off, kDenseTN, (sg.rows + 31) / 32}.store(i, o, v);
  }
}

// ---------------------------------------------------------------- SIMT GEMMs
// 64 x 64 tile, 256 threads with 4 x 4 outputs each, K staged 16 at a time
// (the FP64 build, where the tensor cores' TF32 path does not apply).
constexpr int kSimtTile = 64;

template <typename R, typename Op>
__device__ __forceinline__ void simt_tile(const Op& op, int kpad, int m_valid, int n_valid) {
  constexpr int T = kSimtTile, TK = 16;
  __shared__ R sA[TK][T];
  __shared__ R sB[TK][T];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  R acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = 0;
  for (int k0 = 0; k0 < kpad; k0 += TK) {
    // 64 rows x 4 chunks of 4 K values per operand: one chunk per thread
    {
      const int row = threadIdx.x >> 2, c = threadIdx.x & 3, k = k0 + 4 * c;
      V4<R> va, vb;
      va.x = va.y = va.z = va.w = 0;
      vb = va;
      if (k < kpad && row < m_valid) va = op.load_a(k, row);
      if (k < kpad && row < n_valid) vb = op.load_b(k, row);
      sA[4 * c][row] = va.x; sA[4 * c + 1][row] = va.y; sA[4 * c + 2][row] = va.z; sA[4 * c + 3][row] = va.w;
      sB[4 * c][row] = vb.x; sB[4 * c + 1][row] = vb.y; sB[4 * c + 2][row] = vb.z; sB[4 * c + 3][row] = vb.w;
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
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] += av[p] * bv[q];
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const int i = ty * 4 + p;
    if (i >= m_valid) continue;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = tx * 4 + q;
      if (j < n_valid) op.store(i, j, acc[p][q]);
    }
  }
}

template <typename R, int BWD>
__global__ void __launch_bounds__(256) ms_ctrl_gemm_simt_kernel(MsArgs<R> a, const DenseJob* jobs, int kslot) {
  const DenseJob jb = jobs[blockIdx.x];
  int m_valid, n_valid, kpad;
  if (BWD) {
    const BwdOperands<R> op = bwd_operands<R>(a, jb, kslot, m_valid, n_valid, kpad, kSimtTile, kSimtTile);
    simt_tile<R>(op, kpad, m_valid, n_valid);
  } else {
    const FwdOperands<R> op = fwd_operands<R>(a, jb, kslot, m_valid, n_valid, kpad, kSimtTile, kSimtTile);
    simt_tile<R>(op, kpad, m_valid, n_valid);
  }
}

// ------------------------------------------------------- transposed weights
// W_l^T of every (robot, layer) block listed in segs: WT[i][o] = W[o][i] for
// i < cols, o < rows; rows of WT padded to wt_pitch (pad entries stay zero).

template <typename R>
__global__ void __launch_bounds__(256) ms_transpose_weights_kernel(const R* __restrict__ w, R* __restrict__ wt,
                                                                  const TransSeg* segs, int n_segs) {
  __shared__ R tile[32][33];
  int sidx = 0;
  for (int q = 1; q < n_segs; ++q)
    if ((int)blockIdx.x >= segs[q].tile0) sidx = q;
  const TransSeg sg = segs[sidx];
  const int t = blockIdx.x - sg.tile0;
  const int tiles_c = (sg.cols + 31) / 32;
  const int r0 = (t / tiles_c) * 32, c0 = (t % tiles_c) * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int y = ty; y < 32; y += 8) {
    const int r = r0 + y, c = c0 + tx;
    tile[y][tx] = (r < sg.rows && c < sg.cols) ? w[sg.w_off + (size_t)r * sg.pitch + c] : R(0);
  }
  __syncthreads();
  for (int y = ty; y < 32; y += 8) {
    const int c = c0 + y, r = r0 + tx;
    if (c < sg.cols && r < sg.rows) wt[sg.wt_off + (size_t)c * sg.wt_pitch + r] = tile[tx][y];
  }
}

}  // namespace cls
