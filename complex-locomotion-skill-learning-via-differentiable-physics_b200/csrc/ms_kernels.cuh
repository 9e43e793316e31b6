// ms_kernels.cuh -- fused mass-spring + MLP-controller segment kernels.
//
// One CTA owns one environment (a robot instance) at a time and advances it
// through a whole segment of substeps with the state resident in shared memory,
// so a substep costs no kernel launch and no global round trip of the state.
// Environments are independent in the forward pass (the reference couples them
// only through the shared weights, which are read-only here), so CTAs never
// synchronise with one another.  Per substep, for the env it owns, a CTA runs
// the reference's chain
//   compute_center / compute_height / compute_rotation
//     (multitask/solver_mass_spring.py:150-192)
//   nn_input (multitask/taichi_env.py:149-183)
//   Model.nn1 / nn2 (multitask/nn.py:130-146), generalised to L layers
//   apply_spring_force (multitask/solver_mass_spring.py:86-105)
//   advance_toi (multitask/solver_mass_spring.py:117-148)
// and the reverse kernel replays the hand-written adjoint of that chain in
// reverse order (what ti.ad.Tape does for multitask/diffphy_trainer.py:246-256).
//
// Spring forces are gathered per vertex from a CSR incidence list (springs
// sorted by endpoint) instead of scattered with atomics: every vertex sums its
// own incident impulses in a fixed order, so v_inc needs no atomics and the
// checkpoint recompute reproduces the first pass bit for bit.
#pragma once
#include "cls_common.cuh"

namespace cls {

struct RobotDesc {
  int n_v, n_s, n_out, n_c;          // vertices, springs, MLP outputs, compact inputs
  int ptr_off;                       // CSR row pointers start (n_v + 1 entries)
  int inc_off;                       // incidence entries start (2 n_s entries)
  int spr_off;                       // per-spring output map start (n_s entries)
  int robot_id;                      // 100 selects the hard-coded heading vertices
  int pos_pad;                       // first compact column after the position block
  int n_layers;
  int width[kMaxLayers + 1];         // width[0] = n_c ... width[n_layers] = n_out
  int pitch[kMaxLayers];             // row pitch (elements, multiple of 4) of layer l
  long long w_off[kMaxLayers];       // compact weight offsets (elements)
  int b_off[kMaxLayers];             // bias offsets
  int n_env;                         // envs of this type in this handle
  int loss_envs;                     // B in the loss normalisation (n_env unless a rank holds
                                     // one shard of a controller's envs: cls_set_loss_envs)
  int env_first;                     // envs are sorted by type
  int rot_idx[4];                    // heading vertices for robot 100
};

// Batched-controller offsets of one robot type, kept out of RobotDesc (which
// the fused kernels hold in shared memory) so that the fused kernels' shared
// footprint does not grow with them.
struct DenseDesc {
  long long wt_off[kMaxLayers];      // transposed compact weights
  int wt_pitch[kMaxLayers];          // row pitch of W_l^T: width[l + 1] padded to 4
  // FP32: offsets in `tiles` of the pre-split operand tiles of layer l's
  // forward GEMM (A: inputs of the type's envs, B: W_l) and adjoint GEMM
  // (A: dZ_l, B: W_l^T)
  long long ta_f[kMaxLayers], tb_f[kMaxLayers], ta_b[kMaxLayers], tb_b[kMaxLayers];
  // FP32 weight-gradient products of a segment, offsets in `wtiles`: dZ_l^T
  // (rows = outputs, tile 128) and A_l^T plus a row of ones (rows = inputs + 1,
  // tile 64), K = (record slot, env) with the envs padded to nep (a multiple
  // of 32) and nkt_w K blocks of 32 allocated
  long long tw_d[kMaxLayers], tw_a[kMaxLayers];
  int nep, nkt_w;
};

// one (robot, layer, operand) source of the per-segment transposes for the
// weight-gradient products
struct WgTrans {
  int robot, layer;
  int kind;   // 0: inputs (rec_in), 1: act(rec_z of layer - 1 + bias), 2: dZ (rec_dz)
  int cols;   // valid columns; kinds 0/1 add a row of ones at `cols`
};
// column tile c0 .. c0 + 31 of transpose job `job`
struct WgCol {
  int job, c0;
};
// one output tile (outputs o0 .., inputs i0 ..) of layer l's weight gradient,
// K split `split` of `nsplit`
struct WgJob {
  int robot, layer, o0, i0, split, nsplit;
};

// one output tile of one layer's GEMM: envs [m0, m0 + tile) of robot `robot`
// (env index within the type), outputs [n0, n0 + tile)
struct DenseJob {
  int robot, layer, m0, n0;
};

// one (robot, layer) block of the pre-split weight packing
struct SplitSeg {
  long long w_off, tf_off, tb_off;
  int rows, cols, pitch;  // W_l: rows = outputs, cols = inputs
  long long first;        // first weight of this block in the launch
};

// one (robot, layer) block of the W_l^T transpose (FP64 batched path)
struct TransSeg {
  long long w_off, wt_off;
  int rows, cols, pitch, wt_pitch;
  int tile0;  // first 32 x 32 tile of this block in the launch
};

struct EnvDesc {
  int robot;
  int v_off;                         // vertex offset in packed state arrays
  int in_off;                        // offset in the compact-input record slab
  int z_off[kMaxLayers];             // offset in each layer's record slab
};

template <typename R>
struct MsArgs {
  // sizes and constants
  int n_envs, T, steps, K;           // trajectory length, episode steps, checkpoint interval
  int rec_from;                      // FWD_RECTAIL: first substep the first pass records
  int n_items;                       // work items (entries of `order`) in this launch
  int n_sin, dup_v, dup_h, dup_c;
  int act_hidden, act_out;
  int run_period, turn_period, jump_period;
  int loss_mask;
  int v_total, in_total;
  int z_total[kMaxLayers];
  long long z_base[kMaxLayers];      // layer offsets inside rec_z / rec_dz (per-step slab * K)
  // shared-memory capacities (elements): vertices, compact input (pitch 0),
  // layer outputs (max of hidden widths and n_out, padded to 4), reverse
  // buffer A (max of outputs and the position block), MLP outputs alone
  int smem_nmax, smem_p0max, smem_dmax, smem_amax, smem_omax;
  // controller in shared memory for the whole item (fused kernels, robots
  // small enough): capacities of the weight and bias copies in elements;
  // 0: weights and biases are read from global memory every substep
  int w_smem, b_smem;
  R dt, gravity, ground, drag_s, dashpot, friction, max_speed;
  // tables
  const RobotDesc* robots;
  const EnvDesc* envs;
  const int* order;                  // env processing order (largest first)
  // per-env windows (serving): win[e] = {t_begin, t_end, source checkpoint,
  // first reverse segment}; nullptr: the launch's own arguments for all envs
  const int4* win;
  const int* env_steps;              // per-env episode steps (nullptr: steps)
  int* queue;                        // work-queue counter, zeroed before each launch
  const int* inc_ptr;                // CSR row pointers (relative to inc_off)
  const int4* inc_i;                 // {other vertex, side (0: a, 1: b), spring, out index}
  const V4<R>* inc_f;                // {rest length, stiffness, actuation coef, 0}
  const int4* inc_p;                 // FP32 only: packed 16-byte incidence records
  const int* spring_out;             // per spring: MLP output index or -1
  const int4* spr_ab;                // per spring {a, b, MLP output or -1, 0} (spr_off)
  const V4<R>* spr_p;                // per spring {rest length, stiffness, actuation coef, 0}
  int imp_cap;                       // springs of the shared impulse table (0: none)
  int adj_cap;                       // springs of the shared adjoint table (0: none; the
                                     // batched step kernels keep their occupancy instead)
  const R* w;                        // compact weights
  const R* bias;
  const R* sin_table;                // [T + 1][n_sin], sin(omega (t) dt + 2 pi j / n_sin)
  // state
  V4<R>* ckpt_x; V4<R>* ckpt_v;      // [n_ckpt][v_total]
  V4<R>* fin_x; V4<R>* fin_v;        // [v_total] state after the last processed step
  V4<R>* rec_x; V4<R>* rec_v;        // [K][v_total]
  V4<R>* rec_vinc;                   // [K][v_total] v_inc[t] of the recompute
  R* rec_in;                         // [K][in_total]
  R* rec_z;                          // per layer z_base[l] + [K][z_total[l]]
  R* rec_dz;                         // same layout as rec_z
  unsigned char* head;               // [v_total] head/tail split at t = 0
  // observables, [T][n_envs] (zero where the reference never writes them)
  V4<R>* obs_center; R* obs_height; R* obs_upper; R* obs_rot;
  V4<R>* x_full;                     // [T][v_total] or null
  R* act_full;                       // [T][z_total[L-1]] or null
  // targets [T][n_envs]
  const V4<R>* tv; const R* th; const R* tc;
  const V4<R>* init_obj;             // [v_total] initial_objects per env (pose loss)
  // adjoint carries between segments
  V4<R>* adj_x; V4<R>* adj_v; R* adj_h;
  // batched controller: state between step launches, d input positions
  // [v_total][3], transposed compact weights
  V4<R>* live_x; V4<R>* live_v; R* din; const R* wt;
  R* tiles;                          // FP32: pre-split GEMM operand tiles
  R* wtiles;                         // FP32: weight-gradient operand tiles (one segment)
  const DenseDesc* dense;            // per robot type
  // status
  int* status;
  // tensor-core tiles: poll limit of their waits (0: default) and the
  // bounded-wait self-test (cls_debug_gemm_starve)
  unsigned gemm_wait_limit;
  int gemm_starve;
  // per-phase clock totals, only written by builds with CLS_PHASE_TIMERS
  unsigned long long* phase;
};

// Optional phase timers (profiling builds only, -DCLS_PHASE_TIMERS): thread 0
// of every CTA adds the clock64 time since the previous mark to phase[k].
#ifdef CLS_PHASE_TIMERS
#define CLS_PHASE_START() long long cls_pt_ = clock64()
#define CLS_PHASE(a, k)                                                        \
  do {                                                                         \
    if (threadIdx.x == 0 && (a).phase) {                                       \
      const long long n_ = clock64();                                          \
      atomicAdd((a).phase + (k), (unsigned long long)(n_ - cls_pt_));          \
      cls_pt_ = n_;                                                            \
    }                                                                          \
  } while (0)
#else
#define CLS_PHASE_START() \
  do {                    \
  } while (0)
#define CLS_PHASE(a, k) \
  do {                  \
  } while (0)
#endif

// ------------------------------------------------------------ shared memory
// reduction scratch: 8 values x 32 warps, then 32 ints for arg-reductions;
// the forward pass's fused observable reduction (11 sums and two extrema with
// their indices per warp) takes kRedFwd.  The reverse pass keeps kRed: with
// its packed vertex rows its shared memory (155 KB for the largest
// benchmark robot) sits under the 164 KB carveout step.
constexpr int kRed = 320;
constexpr int kRedFwd = 512;
constexpr int kRedInt = 256;
template <typename R>
struct FwdSmem {
  V4<R>* xs; V4<R>* vs; V4<R>* vinc;
  R* ain;          // compact input, padded
  R* buf0; R* buf1;
  R* red;          // kRedFwd entries
  unsigned char* head;  // per-vertex heading side (rotation of robots other than 100)
  V4<R>* imp;      // per-spring impulses when MsArgs::imp_cap > 0, else null
  R* w; R* b;      // the env's controller when MsArgs::w_smem > 0, else null
};

template <typename R>
__device__ __forceinline__ FwdSmem<R> carve_fwd(char* base, const MsArgs<R>& a) {
  FwdSmem<R> s;
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base + off; off += (bytes + 255) & ~size_t(255); return p; };
  s.xs = (V4<R>*)take(sizeof(V4<R>) * a.smem_nmax);
  s.vs = (V4<R>*)take(sizeof(V4<R>) * a.smem_nmax);
  s.vinc = (V4<R>*)take(sizeof(V4<R>) * a.smem_nmax);
  s.ain = (R*)take(sizeof(R) * a.smem_p0max);
  s.buf0 = (R*)take(sizeof(R) * a.smem_dmax);
  s.buf1 = (R*)take(sizeof(R) * a.smem_dmax);
  s.red = (R*)take(sizeof(R) * kRedFwd);
  s.head = (unsigned char*)take(a.smem_nmax);
  s.imp = a.imp_cap ? (V4<R>*)take(sizeof(V4<R>) * a.imp_cap) : nullptr;
  s.w = a.w_smem ? (R*)take(sizeof(R) * a.w_smem) : nullptr;
  s.b = a.w_smem ? (R*)take(sizeof(R) * a.b_smem) : nullptr;
  return s;
}

// shared memory of the controller copy (weights, then biases)
template <typename R>
__host__ __device__ inline size_t ctrl_smem_bytes(long long w_elems, long long b_elems) {
  auto rb = [](size_t b) { return (b + 255) & ~size_t(255); };
  return w_elems > 0 ? rb(sizeof(R) * (size_t)w_elems) + rb(sizeof(R) * (size_t)b_elems) : 0;
}

template <typename R>
__host__ __device__ inline size_t fwd_smem_bytes(int nmax, int dmax, int p0max, size_t imp_cap) {
  auto rb = [](size_t b) { return (b + 255) & ~size_t(255); };
  return 3 * rb(sizeof(V4<R>) * nmax) + rb(sizeof(R) * p0max) + 2 * rb(sizeof(R) * dmax) +
         rb(sizeof(R) * kRedFwd) + rb(nmax) + (imp_cap ? rb(sizeof(V4<R>) * imp_cap) : 0);
}

// Two 3-vectors p, q of a vertex in 6 values of shared memory: lo[i] =
// {p.x, p.y, p.z, q.x} (one 16-byte access in FP32), hi[i] = {q.y, q.z} (one
// 8-byte access).  A row costs 24 bytes instead of two 16-byte rows, with the
// same number of shared-memory accesses when both vectors are read.
template <typename R>
struct alignas(2 * sizeof(R)) V2 {
  R x, y;
};
template <typename R>
struct PairRows {
  V4<R>* lo;
  V2<R>* hi;
  __device__ __forceinline__ V4<R> p(int i) const {
    V4<R> u = lo[i];
    u.w = 0;
    return u;
  }
  __device__ __forceinline__ void get(int i, V4<R>& pv, V4<R>& qv) const {
    const V4<R> u = lo[i];
    const V2<R> h = hi[i];
    pv.x = u.x; pv.y = u.y; pv.z = u.z; pv.w = 0;
    qv.x = u.w; qv.y = h.x; qv.z = h.y; qv.w = 0;
  }
  __device__ __forceinline__ void set(int i, const V4<R>& pv, const V4<R>& qv) const {
    V4<R> u;
    u.x = pv.x; u.y = pv.y; u.z = pv.z; u.w = qv.x;
    V2<R> h;
    h.x = qv.y; h.y = qv.z;
    lo[i] = u;
    hi[i] = h;
  }
  // p of row i += d (q unchanged)
  __device__ __forceinline__ void add_p(int i, R d0, R d1, R d2) const {
    V4<R> u = lo[i];
    u.x += d0; u.y += d1; u.z += d2;
    lo[i] = u;
  }
};

// Reverse-pass shared memory.  xv holds x(t), v(t) of the substep being
// reversed, g the adjoint state (d x, d v).  io holds the controller outputs
// [0, omax) and d loss / d output [obuf, obuf + omax) up to the output layer's
// dz, then the transposed products (d loss / d layer input; 3 N position
// columns for layer 0).  gvinc (v_inc, then its adjoint) is live only from
// the v_inc recompute to the end of the spring adjoint; dz and part are live
// only in the MLP adjoint that follows, so they share one region.
template <typename R>
struct RevSmem {
  PairRows<R> xv, g;
  R* bufA;         // controller outputs, then the transposed products
  R* bufB;         // d loss / d output (inside the same region as bufA)
  V4<R>* gvinc;    // union region, vertex phase
  R* dz;           // union region, MLP phase
  V4<R>* part;     // union region, MLP phase: blockDim partials
  R* red;
  V4<R>* adj;      // per-spring adjoint terms (2 per spring) when MsArgs::adj_cap > 0
  R* w; R* b;      // the env's controller when MsArgs::w_smem > 0, else null
};

template <typename R>
__host__ __device__ inline size_t rev_union_bytes(int nmax, int dmax, int threads) {
  auto rb = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t vert = rb(sizeof(V4<R>) * nmax);
  const size_t mlp = rb(sizeof(R) * dmax) + rb(sizeof(V4<R>) * threads);
  return vert > mlp ? vert : mlp;
}

// offset of d loss / d output inside the outputs / products region, and the
// region's size in values
__host__ __device__ inline int rev_obuf(int omax) { return (omax + 63) & ~63; }
__host__ __device__ inline int rev_io_values(int amax, int omax) {
  const int o2 = rev_obuf(omax) + omax;
  return amax > o2 ? amax : o2;
}

template <typename R>
__device__ __forceinline__ RevSmem<R> carve_rev(char* base, const MsArgs<R>& a) {
  RevSmem<R> s;
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = base + off; off += (bytes + 255) & ~size_t(255); return p; };
  s.xv.lo = (V4<R>*)take(sizeof(V4<R>) * a.smem_nmax);
  s.xv.hi = (V2<R>*)take(sizeof(V2<R>) * a.smem_nmax);
  s.g.lo = (V4<R>*)take(sizeof(V4<R>) * a.smem_nmax);
  s.g.hi = (V2<R>*)take(sizeof(V2<R>) * a.smem_nmax);
  s.bufA = (R*)take(sizeof(R) * rev_io_values(a.smem_amax, a.smem_omax));
  s.bufB = s.bufA + rev_obuf(a.smem_omax);
  s.red = (R*)take(sizeof(R) * kRed);
  char* u = take(rev_union_bytes<R>(a.smem_nmax, a.smem_dmax, blockDim.x));
  s.gvinc = (V4<R>*)u;
  s.dz = (R*)u;
  s.part = (V4<R>*)(u + ((sizeof(R) * a.smem_dmax + 255) & ~size_t(255)));
  s.adj = a.adj_cap ? (V4<R>*)take(2 * sizeof(V4<R>) * a.adj_cap) : nullptr;
  s.w = a.w_smem ? (R*)take(sizeof(R) * a.w_smem) : nullptr;
  s.b = a.w_smem ? (R*)take(sizeof(R) * a.b_smem) : nullptr;
  return s;
}

template <typename R>
__host__ __device__ inline size_t rev_smem_bytes(int nmax, int amax, int omax, int dmax, int threads,
                                                size_t adj_cap) {
  auto rb = [](size_t b) { return (b + 255) & ~size_t(255); };
  return 2 * (rb(sizeof(V4<R>) * nmax) + rb(sizeof(V2<R>) * nmax)) + rb(sizeof(R) * rev_io_values(amax, omax)) +
         rb(sizeof(R) * kRed) + rev_union_bytes<R>(nmax, dmax, threads) +
         (adj_cap ? rb(2 * sizeof(V4<R>) * adj_cap) : 0);
}

// ------------------------------------------------------------- primitives

// Hooke + dashpot impulse of one spring seen from one of its endpoints
// (solver_mass_spring.py:89-103).  xa/xb/va/vb are the spring's a/b endpoints.
template <typename R>
__device__ __forceinline__ void spring_impulse(const V4<R>& xa, const V4<R>& xb, const V4<R>& va,
                                               const V4<R>& vb, R l0, R k, R coef, R act, R dt,
                                               R dashpot, R imp[3]) {
  R d0 = xa.x - xb.x, d1 = xa.y - xb.y, d2 = xa.z - xb.z;
  R n2 = d0 * d0 + d1 * d1 + d2 * d2;
  R length = sqrt_s<R>(n2 + R(1e-8)) + R(1e-4);        // norm(1e-8) + 1e-4
  R target = l0 * (R(1) + coef * act);
  R sc = dt * (length - target) * k * rcp_s<R>(length);
  R invlen = rsqrt_s<R>(n2);                           // normalized(): 1 / norm()
  R n0 = d0 * invlen, n1 = d1 * invlen, nz = d2 * invlen;
  R vrel = (va.x - vb.x) * n0 + (va.y - vb.y) * n1 + (va.z - vb.z) * nz;
  R c = dashpot * vrel;
  imp[0] = sc * d0 + c * n0;
  imp[1] = sc * d1 + c * n1;
  imp[2] = sc * d2 + c * nz;
}

// One spring incidence: the other endpoint, which side this vertex is on, the
// controller output driving the spring, and the spring constants.
template <typename R>
struct Inc {
  int other, side, out;
  R l0, k, coef;
};

// FP32 records are packed in 16 bytes: {other | side << 15 | (out + 1) << 16,
// l0, k, coef}; FP64 records use the two-array form (int4 + V4<double>).
template <typename R>
__device__ __forceinline__ Inc<R> load_inc(const MsArgs<R>& a, const RobotDesc& rb, int q,
                                           unsigned long long pol);
template <>
__device__ __forceinline__ Inc<float> load_inc<float>(const MsArgs<float>& a, const RobotDesc& rb,
                                                      int q, unsigned long long pol) {
  const int4 p = ldg_i4_hint(a.inc_p + rb.inc_off + q, pol);
  Inc<float> r;
  r.other = p.x & 0x7fff;
  r.side = (p.x >> 15) & 1;
  r.out = (int)(((unsigned)p.x) >> 16) - 1;
  r.l0 = __int_as_float(p.y);
  r.k = __int_as_float(p.z);
  r.coef = __int_as_float(p.w);
  return r;
}
template <>
__device__ __forceinline__ Inc<double> load_inc<double>(const MsArgs<double>& a, const RobotDesc& rb,
                                                        int q, unsigned long long pol) {
  const int4 ii = ldg_i4_hint(a.inc_i + rb.inc_off + q, pol);
  const V4<double> ff = ldg4_hint<double>(a.inc_f + rb.inc_off + q, pol);
  Inc<double> r;
  r.other = ii.x; r.side = ii.y; r.out = ii.w;
  r.l0 = ff.x; r.k = ff.y; r.coef = ff.z;
  return r;
}

template <typename R>
__device__ __forceinline__ void accumulate_incidence(const MsArgs<R>& a, const Inc<R>& in, const V4<R>& xi,
                                                     const V4<R>& vi, const V4<R>* xs, const V4<R>* vs,
                                                     const R* out, R& s0, R& s1, R& s2) {
  const int o = in.other;
  const R act = in.out >= 0 ? out[in.out] : R(0);
  R imp[3];
  if (in.side == 0) {  // this vertex is endpoint a: -impulse
    spring_impulse<R>(xi, xs[o], vi, vs[o], in.l0, in.k, in.coef, act, a.dt, a.dashpot, imp);
    s0 -= imp[0]; s1 -= imp[1]; s2 -= imp[2];
  } else {             // endpoint b: +impulse
    spring_impulse<R>(xs[o], xi, vs[o], vi, in.l0, in.k, in.coef, act, a.dt, a.dashpot, imp);
    s0 += imp[0]; s1 += imp[1]; s2 += imp[2];
  }
}

// v_inc of all vertices, half-warp per vertex: the 16 lanes of a half-warp
// take the vertex's incidences in parallel (lane l: entries beg + l, beg + l +
// 16, ...) and combine them with a fixed xor-shuffle tree, so the result does
// not depend on scheduling (the recompute pass reproduces the first pass bit
// for bit).  Each half-warp prefetches the first incidence of U vertices
// before computing, so U records per lane are in flight.
#ifndef CLS_GATHER_U
#define CLS_GATHER_U 4
#endif
template <typename R>
__device__ __forceinline__ void gather_vinc_all(const MsArgs<R>& a, const RobotDesc& rb, int N,
                                                const V4<R>* xs, const V4<R>* vs, const R* out,
                                                V4<R>* vinc, V4<R>* rec) {
  constexpr int U = CLS_GATHER_U;
  const unsigned long long pol = policy_evict_last();
  const int lane = threadIdx.x & 31, wid = (threadIdx.x >> 5), nw = (blockDim.x >> 5);
  const int l16 = lane & 15, half = lane >> 4;
  const int* ptr = a.inc_ptr + rb.ptr_off;
  const int stride = nw * 2;
  // the loop bound is warp-uniform (vb0), so both half-warps run the same
  // iterations and every full-mask shuffle below has all 32 lanes
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
      R s0 = 0, s1 = 0, s2 = 0;
      if (v < N) {
        const V4<R> xi = xs[v], vi = vs[v];
        int q = beg[k] + l16;
        if (q < end[k]) accumulate_incidence<R>(a, first[k], xi, vi, xs, vs, out, s0, s1, s2);
        for (q += 16; q < end[k]; q += 16)
          accumulate_incidence<R>(a, load_inc<R>(a, rb, q, pol), xi, vi, xs, vs, out, s0, s1, s2);
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      }
      if (l16 == 0 && v < N) {
        V4<R> r; r.x = s0; r.y = s1; r.z = s2; r.w = 0;
        vinc[v] = r;
        if (rec) rec[v] = r;
      }
    }
  }
}

// The same v_inc with each spring's impulse computed once: phase A evaluates
// every spring (spring-parallel, a -> b order as both of its incidences do) into
// imp[], phase B is gather_vinc_all's half-warp gather with the impulses read
// from imp[] instead of recomputed, in the same lanes and the same order.  For
// robots whose impulse table fits in shared memory (MsArgs::imp_cap).
// spring-parallel table phase: the next spring's records in flight while one
// is evaluated (spider step kernel, 4096 envs: forward 11.65 -> 11.41 ms per
// 61 substeps)
#ifndef CLS_TABLE_PREFETCH
#define CLS_TABLE_PREFETCH 1
#endif
template <typename R>
__device__ __forceinline__ void gather_vinc_table(const MsArgs<R>& a, const RobotDesc& rb, int N,
                                                  const V4<R>* xs, const V4<R>* vs, const R* out,
                                                  V4<R>* imp, V4<R>* vinc, V4<R>* rec) {
  constexpr int U = 4;
  const unsigned long long pol = policy_evict_last();
  const int tid = threadIdx.x, nt = blockDim.x;
#if CLS_TABLE_PREFETCH
  // the next spring's records are loaded before this one is evaluated, so
  // one pair of L2 loads per thread is always in flight (same arithmetic)
  int4 ab = make_int4(0, 0, -1, 0);
  V4<R> f;
  f.x = f.y = f.z = f.w = R(0);
  if (tid < rb.n_s) {
    ab = ldg_i4_hint(a.spr_ab + rb.spr_off + tid, pol);
    f = ldg4_hint<R>(a.spr_p + rb.spr_off + tid, pol);
  }
  for (int sp = tid; sp < rb.n_s; sp += nt) {
    const int nx = sp + nt;
    int4 ab_n = ab;
    V4<R> f_n = f;
    if (nx < rb.n_s) {
      ab_n = ldg_i4_hint(a.spr_ab + rb.spr_off + nx, pol);
      f_n = ldg4_hint<R>(a.spr_p + rb.spr_off + nx, pol);
    }
    const R act = ab.z >= 0 ? out[ab.z] : R(0);
    R im[3];
    spring_impulse<R>(xs[ab.x], xs[ab.y], vs[ab.x], vs[ab.y], f.x, f.y, f.z, act, a.dt, a.dashpot, im);
    V4<R> r; r.x = im[0]; r.y = im[1]; r.z = im[2]; r.w = 0;
    imp[sp] = r;
    ab = ab_n;
    f = f_n;
  }
#else
  for (int sp = tid; sp < rb.n_s; sp += nt) {
    const int4 ab = ldg_i4_hint(a.spr_ab + rb.spr_off + sp, pol);
    const V4<R> f = ldg4_hint<R>(a.spr_p + rb.spr_off + sp, pol);
    const R act = ab.z >= 0 ? out[ab.z] : R(0);
    R im[3];
    spring_impulse<R>(xs[ab.x], xs[ab.y], vs[ab.x], vs[ab.y], f.x, f.y, f.z, act, a.dt, a.dashpot, im);
    V4<R> r; r.x = im[0]; r.y = im[1]; r.z = im[2]; r.w = 0;
    imp[sp] = r;
  }
#endif
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = (threadIdx.x >> 5), nw = (blockDim.x >> 5);
  const int l16 = lane & 15, half = lane >> 4;
  const int* ptr = a.inc_ptr + rb.ptr_off;
  const int stride = nw * 2;
  for (int vb0 = wid * 2; vb0 < N; vb0 += stride * U) {
    const int vb = vb0 + half;
    int beg[U], end[U];
    int4 first[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int v = vb + k * stride;
      beg[k] = 0;
      end[k] = 0;
      if (v < N) { beg[k] = ptr[v]; end[k] = ptr[v + 1]; }
      const int q = beg[k] + l16;
      first[k] = make_int4(0, 0, 0, 0);
      if (q < end[k]) first[k] = ldg_i4_hint(a.inc_i + rb.inc_off + q, pol);
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int v = vb + k * stride;
      R s0 = 0, s1 = 0, s2 = 0;
      if (v < N) {
        int q = beg[k] + l16;
        for (int4 in = first[k]; q < end[k];) {
          const V4<R> im = imp[in.z];
          if (in.y == 0) { s0 -= im.x; s1 -= im.y; s2 -= im.z; }
          else { s0 += im.x; s1 += im.y; s2 += im.z; }
          q += 16;
          if (q < end[k]) in = ldg_i4_hint(a.inc_i + rb.inc_off + q, pol);
        }
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      }
      if (l16 == 0 && v < N) {
        V4<R> r; r.x = s0; r.y = s1; r.z = s2; r.w = 0;
        vinc[v] = r;
        if (rec) rec[v] = r;
      }
    }
  }
}

// advance_toi for one vertex (solver_mass_spring.py:119-148); in place
template <typename R>
__device__ __forceinline__ void advance_vertex(const MsArgs<R>& a, V4<R>& x, V4<R>& v, const V4<R>& vi) {
  R ov0 = a.drag_s * v.x + vi.x;
  R ov1 = a.drag_s * v.y + a.dt * a.gravity + vi.y;
  R ov2 = a.drag_s * v.z + vi.z;
  R nv0 = ov0, nv1 = ov1, nv2 = ov2, toi = 0;
  R nx1 = x.y + a.dt * ov1;
  if (nx1 < a.ground && ov1 < R(-1e-4)) {
    toi = -(x.y - a.ground) / ov1;
    R f = a.friction * (-ov1);
    nv1 = 0;
    nv0 = (ov0 < 0) ? fmin(R(0), ov0 + f) : fmax(R(0), ov0 - f);
    nv2 = (ov2 < 0) ? fmin(R(0), ov2 + f) : fmax(R(0), ov2 - f);
  }
  R dtt = a.dt - toi;
  x.x = x.x + toi * ov0 + dtt * nv0;
  x.y = x.y + toi * ov1 + dtt * nv1;
  x.z = x.z + toi * ov2 + dtt * nv2;
  v.x = nv0; v.y = nv1; v.z = nv2;
}

// One 4-wide group of controller weights: from the shared-memory copy (SH) or
// from global memory, not allocated in L1 and evict-first in L2 (pol).
template <typename R, bool SH>
__device__ __forceinline__ V4<R> ldw4(const V4<R>* p, unsigned long long pol) {
  if constexpr (SH) return *p;
  else return ldg4_hint<R>(p, pol);
}

// The env's controller -- weights and biases, each contiguous per robot --
// copied into shared memory (sw, sb) at the start of a work item; the caller
// synchronises before the first product.
template <typename R>
__device__ __forceinline__ void load_controller_smem(const R* __restrict__ w, const R* __restrict__ bias,
                                                     const RobotDesc& rb, R* sw, R* sb) {
  const int L = rb.n_layers;
  const long long w0 = rb.w_off[0];
  const long long n4 = (rb.w_off[L - 1] + (long long)rb.width[L] * rb.pitch[L - 1] - w0) >> 2;
  const V4<R>* src = reinterpret_cast<const V4<R>*>(w + w0);
  V4<R>* dst = reinterpret_cast<V4<R>*>(sw);
  for (long long i = threadIdx.x; i < n4; i += blockDim.x) dst[i] = ldg4<R>(src + i);
  const int b0 = rb.b_off[0], nb = rb.b_off[L - 1] + ((rb.width[L] + 3) & ~3) - b0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) sb[i] = bias[b0 + i];
}

#ifndef CLS_GEMV_UNROLL
#define CLS_GEMV_UNROLL 2
#endif
constexpr int kGemvUnroll = CLS_GEMV_UNROLL;
// y = act(W x + b) for one layer.  Each warp owns RB consecutive rows at a
// time and streams them together (RB independent float4 loads per lane per
// column step), so short rows -- the 128-wide output layer of a robot with
// thousands of actuators -- still keep enough loads in flight.
// Records z (pre-bias sums) when zrec != null.
template <typename R, int RB, bool SH>
__device__ __forceinline__ void dense_forward_rb(const R* __restrict__ W, int pitch, int nout,
                                                 const R* __restrict__ bias, const R* xin, R* y,
                                                 R* zrec, int act) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int n4 = pitch >> 2;
  const V4<R>* x4 = reinterpret_cast<const V4<R>*>(xin);
  const unsigned long long pol = policy_evict_first();
  for (int i0 = wid * RB; i0 < nout; i0 += nw * RB) {
    const V4<R>* w4[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) {
      const int row = (i0 + r < nout) ? i0 + r : i0;
      w4[r] = reinterpret_cast<const V4<R>*>(W + (size_t)row * pitch);
    }
    R s[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) s[r] = 0;
#pragma unroll kGemvUnroll
    for (int j = lane; j < n4; j += 32) {
      const V4<R> xv = x4[j];
      V4<R> wv[RB];
#pragma unroll
      for (int r = 0; r < RB; ++r) wv[r] = ldw4<R, SH>(w4[r] + j, pol);
#pragma unroll
      for (int r = 0; r < RB; ++r)
        s[r] += wv[r].x * xv.x + wv[r].y * xv.y + wv[r].z * xv.z + wv[r].w * xv.w;
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s[r] += __shfl_xor_sync(0xffffffffu, s[r], o);
    }
    if (lane < RB && i0 + lane < nout) {
      R v = s[0];
#pragma unroll
      for (int r = 1; r < RB; ++r)
        if (lane == r) v = s[r];
      const int i = i0 + lane;
      if (zrec) zrec[i] = v;
      y[i] = act_f<R>(act, v + bias[i]);
    }
  }
}

// rows per warp of the controller's products: RB_NARROW for rows of at most
// 256 inputs, RB_WIDE above.  Measured on the 512-robot uneven batch (151
// substeps, first pass + recompute + reverse): RB_WIDE 4 -> 8 took the
// forward launches 25.3 -> 24.3 ms; unrolling the column loop 4 instead of 2
// changed nothing; RB_NARROW 16 measured within noise of 8 and spills in the
// 512-thread instance, so 8 stays
#ifndef CLS_GEMV_RB_NARROW
#define CLS_GEMV_RB_NARROW 8
#endif
#ifndef CLS_GEMV_RB_WIDE
#define CLS_GEMV_RB_WIDE 8
#endif
template <typename R, bool SH>
__device__ __forceinline__ void dense_forward(const R* __restrict__ W, int pitch, int nout,
                                              const R* __restrict__ bias, const R* xin, R* y,
                                              R* zrec, int act) {
  if (pitch <= 256) dense_forward_rb<R, CLS_GEMV_RB_NARROW, SH>(W, pitch, nout, bias, xin, y, zrec, act);
  else dense_forward_rb<R, CLS_GEMV_RB_WIDE, SH>(W, pitch, nout, bias, xin, y, zrec, act);
}

#ifndef CLS_TRANS_KMAX
#define CLS_TRANS_KMAX 4
#endif
#ifndef CLS_TRANS_WIDE_UNROLL
#define CLS_TRANS_WIDE_UNROLL 2
#endif
// row loops of the transposed products: wide rows (layer 0) unrolled 2,
// narrow rows 8 (512-robot uneven batch, 151 substeps, reverse launches:
// narrow 2 / 4 / 8 = 35.8 / 30.7 / 28.7 ms; wide 4 instead of 2: 30.6 ms)
#ifndef CLS_TRANS_NARROW_UNROLL
#define CLS_TRANS_NARROW_UNROLL 8
#endif
constexpr int kTransWideUnroll = CLS_TRANS_WIDE_UNROLL;
constexpr int kTransNarrowUnroll = CLS_TRANS_NARROW_UNROLL;
// g_in[j] = sum_i W[i, j] dz[i] for j in [0, ncols) (ncols multiple of 4 or
// padded), deterministic: fixed row splits, fixed reduction order.
// Result written to out4[j/4] (V4 groups).  Uses `part` (blockDim entries) as
// scratch in the narrow-row case.
template <typename R, bool SH>
__device__ __forceinline__ void dense_transposed(const R* __restrict__ W, int pitch, int nrows,
                                                 int ncols, const R* dz, V4<R>* part, V4<R>* out4) {
  const int c4 = (ncols + 3) >> 2;
  const int tid = threadIdx.x, nt = blockDim.x;
  const unsigned long long pol = policy_evict_first();
  if (nrows == 1) {
    for (int g = tid; g < c4; g += nt) {
      const V4<R> wv = ldw4<R, SH>(reinterpret_cast<const V4<R>*>(W) + g, pol);
      const R d = dz[0];
      V4<R> r; r.x = wv.x * d; r.y = wv.y * d; r.z = wv.z * d; r.w = wv.w * d;
      out4[g] = r;
    }
    __syncthreads();
    return;
  }
  if (2 * c4 > nt) {
    // Wide rows (the first layer of a large robot): two half-blocks split the
    // rows; each thread keeps up to KMAX column-group partials in registers,
    // the first half stores, the second half adds (fixed order).
    constexpr int KMAX = CLS_TRANS_KMAX;
    const int H = nt >> 1, h = tid >= H ? 1 : 0, lt = tid - h * H;
    const int rmid = nrows >> 1, r0 = h ? rmid : 0, r1 = h ? nrows : rmid;
    for (int base = 0; base < c4; base += H * KMAX) {
      R acc[KMAX][4];
#pragma unroll
      for (int k = 0; k < KMAX; ++k) acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0;
#pragma unroll kTransWideUnroll
      for (int i = r0; i < r1; ++i) {
        const R d = dz[i];
        const V4<R>* row = reinterpret_cast<const V4<R>*>(W + (size_t)i * pitch);
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
          const int g = base + lt + k * H;
          if (g < c4) {
            const V4<R> wv = ldw4<R, SH>(row + g, pol);
            acc[k][0] += wv.x * d; acc[k][1] += wv.y * d; acc[k][2] += wv.z * d; acc[k][3] += wv.w * d;
          }
        }
      }
      if (!h) {
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
          const int g = base + lt + k * H;
          if (g < c4) { V4<R> r; r.x = acc[k][0]; r.y = acc[k][1]; r.z = acc[k][2]; r.w = acc[k][3]; out4[g] = r; }
        }
      }
      __syncthreads();
      if (h) {
#pragma unroll
        for (int k = 0; k < KMAX; ++k) {
          const int g = base + lt + k * H;
          if (g < c4) {
            V4<R> r = out4[g];
            r.x += acc[k][0]; r.y += acc[k][1]; r.z += acc[k][2]; r.w += acc[k][3];
            out4[g] = r;
          }
        }
      }
      __syncthreads();
    }
    return;
  }
  // Narrow rows (hidden / output layers): split the rows into `slices`
  // interleaved sets, one partial per thread, then a fixed-order reduction.
  int slices = nt / c4;
  if (slices > nrows) slices = nrows;
  const int used = slices * c4;
  if (tid < used) {
    const int g = tid % c4, r0 = tid / c4;
    R s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll kTransNarrowUnroll
    for (int i = r0; i < nrows; i += slices) {
      const V4<R> wv = ldw4<R, SH>(reinterpret_cast<const V4<R>*>(W + (size_t)i * pitch) + g, pol);
      const R d = dz[i];
      s0 += wv.x * d; s1 += wv.y * d; s2 += wv.z * d; s3 += wv.w * d;
    }
    V4<R> r; r.x = s0; r.y = s1; r.z = s2; r.w = s3;
    part[tid] = r;
  }
  __syncthreads();
  for (int g = tid; g < c4; g += nt) {
    V4<R> acc = part[g];
    for (int r = 1; r < slices; ++r) {
      const V4<R> p = part[r * c4 + g];
      acc.x += p.x; acc.y += p.y; acc.z += p.z; acc.w += p.w;
    }
    out4[g] = acc;
  }
  __syncthreads();
}

template <typename R>
struct MinIdx { R v; int i; };

}  // namespace cls
