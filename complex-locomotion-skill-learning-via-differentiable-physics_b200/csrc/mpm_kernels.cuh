// mpm_kernels.cuh -- differentiable MLS-MPM substep (P2G, grid update, G2P)
// and its hand-written adjoint, dimension-templated (2D / 3D).
//
// Algorithm: the reference's multitask/solver_mpm.py (2D): p2g :83-124,
// grid_op :126-144, g2p :146-165, advance_core_grad :182-190.  Generalised to
// 3D, per-particle fibre directions (actuation stress a * (F f)(F f)^T; the
// reference's is f = e_y) and the compressible neo-Hookean Kirchhoff stress
// mu (F F^T - I) + lambda ln(J) I next to the reference's fixed-corotated
// model (2D only, closed-form polar decomposition).
//
// Layout and kernels (B200):
//  * particles are stored SoA (component planes of E*P values) in an internal
//    order: Morton order of their initial cells, cut into chunks of 256 (one
//    CTA each); inside a chunk the particles are interleaved so that the 32
//    lanes of a warp hold particles of 32 different cells;
//  * the grid is dense per env but blocked: blocks of 4^3 (3D) or 8^2 (2D)
//    nodes, 64 nodes of 4 values (16 B in FP32) per block, so a block is one
//    contiguous 1 KB run.  P2G keeps, per env, the box of the base cells it
//    scattered from (one min/max atomic pair per warp); the grid kernels
//    visit only the blocks under that box, and the accumulators are cleared
//    by the grid kernel that consumes them;
//  * scatters (P2G, G2P^T) go through a warp-private shared-memory tile over
//    the box of the warp's stencils: with distinct base cells per lane, the
//    lanes of one stencil offset write distinct nodes, so the warp adds with
//    plain shared-memory read-modify-writes (a __syncwarp between offsets; a
//    warp whose lanes share a base cell uses shared atomics instead), then
//    flushes each touched node with one 16-byte vector atomic.  Gathers (G2P,
//    P2G^T) read the grid through L1.  A warp whose box exceeds the tile falls
//    back to global atomics;
//  * forward: one fused particle kernel per substep does G2P of step f and
//    P2G of step f + 1 (only x, F and the grid cross kernels; v and C are
//    written when the step is recorded); reverse: one fused kernel does P2G^T
//    and the loss seed of step f, then G2P^T of step f - 1 (only a_x and a_F
//    cross kernels).
#pragma once
#include <climits>

#include "cls_common.cuh"

namespace cls {
namespace mpm {

enum Material : int { FIXED_COROTATED = 0, NEO_HOOKEAN = 1 };

// occupancy targets of the particle kernels (CTAs per SM for the register
// budget); compile-time tuning knobs
#ifndef CLS_MPM_FWD_MIN_BLOCKS
#define CLS_MPM_FWD_MIN_BLOCKS 3
#endif
#ifndef CLS_MPM_ADJ_MIN_BLOCKS
#define CLS_MPM_ADJ_MIN_BLOCKS 2
#endif

constexpr int kChunk = 256;         // particles per CTA, one per thread
constexpr int kWarps = kChunk / 32;
constexpr int kTileDefault = 256;   // default warp tile capacity (nodes)
constexpr int kMaxMuscles = 256;
constexpr int kFwdPlanes = 4;       // staged grid velocity (3) / P2G scatter: momentum (3), mass
constexpr int kAdjPlanes = 6;       // staged grid adjoint (4) / staged velocity (3) + velocity adjoint (3)
// particle-kernel variants (template bitmask): stage the grid a warp gathers
// from in shared memory, scatter through a warp tile
constexpr int kStageGather = 1, kScatterTile = 2;

template <int D>
struct Blk {
  static constexpr int LOG = D == 3 ? 2 : 3;  // block side 4 (3D) or 8 (2D)
  static constexpr int SIDE = 1 << LOG;
  static constexpr int NODES = 64;
};

// Physical constants, body tables and grid geometry shared by all kernels.
template <typename R>
struct Phys {
  int E, P, M, material, n_chunks, tile_cap;  // tile_cap: nodes per warp tile (<= 0: none)
  int n_grid, nb, bound;                      // nodes per side, blocks per side
  long long nblk;                             // blocks per env
  long long EP;                               // E * P (plane stride)
  R dx, inv_dx, dt, ks, mu, la, act_strength, gravity, mass;  // ks = dt p_vol 4 inv_dx^2
  const int* muscle;                          // [P] internal order, -1 passive
  const R* fibre;                             // [D][P]
  const R* pw;                                // [P] particle weights of the centre
  const int* chunk_start;                     // [n_chunks] first internal particle
  const int* chunk_len;                       // [n_chunks] particles (<= kChunk)
  int runs;                                   // 1: base-cell order, run-summed scatters
};

// Forward particle kernel: G2P of step f (mode bit 1) and/or P2G of step g
// (mode bit 2; g = f + 1 after G2P, else the state read from v_in / C_in).
template <typename R>
struct FwdArgs {
  Phys<R> c;
  const R* x_in;          // x_f (with G2P) or x_g (P2G only)
  const V4<R>* gv;        // grid (velocity, mass) of step f
  R* x_out;               // x_{f+1}
  R* v_out;               // v_{f+1} or nullptr
  R* C_out;               // C_{f+1} or nullptr
  const R* v_in;          // v_g, C_g (P2G-only mode)
  const R* C_in;
  const R* F_in;          // F_g
  R* F_out;               // F_{g+1} or nullptr
  const R* act;           // [E][M] of step g
  V4<R>* acc;             // (momentum, mass) accumulator of step g
  int* bbox;              // [E][2 D] box of the base cells of step g (min, max)
  R* csum;                // [E][D] pw-weighted position sums of the positions produced (or read)
};

// Reverse particle kernel: P2G^T of step f plus the loss seed of step f
// (mode bit 1), then G2P^T of step h (mode bit 2; h = f - 1 after P2G^T, else
// the first reverse step h = T - 1 whose x-adjoint is the seed of step T).
template <typename R>
struct AdjArgs {
  Phys<R> c;
  // P2G^T of step f
  const R* x_f; const R* v_f; const R* C_f; const R* F_f;
  const R* act_f;          // [E][M]
  const V4<R>* ga;         // grid adjoint (d velocity, d mass) of step f
  const R* ax_in;          // a_x(f) so far (G2P^T of step f applied)
  const R* aF_in;          // a_F(f + 1)
  R* gact;                 // d actuation [E][M] of step f (accumulated)
  // loss seed of the state whose x-adjoint is completed here
  R seed_w;                // w_t (0: none)
  const R* csum;           // [E][D] pw-weighted position sums of that step
  const R* target;         // [E][D]
  R pw_sum;
  // outputs of the last reverse step (no G2P^T follows)
  R* out_ax; R* out_av; R* out_aC; R* out_aF;
  // G2P^T of step h
  const R* x_h;
  const V4<R>* gv_h;       // grid of step h
  V4<R>* gacc;             // d grid velocity accumulator of step h
  R* ax_out;               // a_x(h) so far
  R* aF_out;               // a_F(f) (zeros in the first reverse step)
};

// ------------------------------------------------------------ helpers
template <typename R, int D>
struct Kern {
  static constexpr int NN = D == 2 ? 9 : 27;

  // quadratic B-spline weights of the 3^D stencil.  The base cell is clamped
  // into [0, n_grid - 3] so that a particle that has left the domain can never
  // address memory outside its env's grid (the reference does not check);
  // for particles inside the domain the clamp has no effect.
  __device__ static void weights(const R* xp, R inv_dx, int n_grid, int base[D], R fx[D], R w[3][D],
                                 R dw[3][D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      base[d] = (int)(xp[d] * inv_dx - R(0.5));
      base[d] = base[d] < 0 ? 0 : (base[d] > n_grid - 3 ? n_grid - 3 : base[d]);
      fx[d] = xp[d] * inv_dx - (R)base[d];
      w[0][d] = R(0.5) * (R(1.5) - fx[d]) * (R(1.5) - fx[d]);
      w[1][d] = R(0.75) - (fx[d] - R(1)) * (fx[d] - R(1));
      w[2][d] = R(0.5) * (fx[d] - R(0.5)) * (fx[d] - R(0.5));
      dw[0][d] = -(R(1.5) - fx[d]);
      dw[1][d] = R(-2) * (fx[d] - R(1));
      dw[2][d] = fx[d] - R(0.5);
    }
  }

  __device__ static void offs(int q, int o[D]) {
    o[0] = q % 3;
    o[1] = (q / 3) % 3;
    if (D == 3) o[D - 1] = q / 9;
  }

  __device__ static R det(const R* A) {
    if (D == 2) return A[0] * A[3] - A[1] * A[2];
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
  }

  __device__ static void cof(const R* A, R* c) {
    if (D == 2) {
      c[0] = A[3]; c[1] = -A[2]; c[2] = -A[1]; c[3] = A[0];
      return;
    }
    c[0] = A[4] * A[8] - A[5] * A[7];
    c[1] = A[5] * A[6] - A[3] * A[8];
    c[2] = A[3] * A[7] - A[4] * A[6];
    c[3] = A[2] * A[7] - A[1] * A[8];
    c[4] = A[0] * A[8] - A[2] * A[6];
    c[5] = A[1] * A[6] - A[0] * A[7];
    c[6] = A[1] * A[5] - A[2] * A[4];
    c[7] = A[2] * A[3] - A[0] * A[5];
    c[8] = A[0] * A[4] - A[1] * A[3];
  }

  // new_F = (I + dt C) F   (solver_mpm.py:89)
  __device__ static void new_F(const R* C, const R* F, R dt, R* nF) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R acc = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) acc += ((i == q ? R(1) : R(0)) + dt * C[i * D + q]) * F[q * D + j];
        nF[i * D + j] = acc;
      }
  }

  // Kirchhoff stress incl. actuation (solver_mpm.py:96-115); `am` is the
  // actuation times its strength, `f` the fibre (active particles only).
  __device__ static void stress(const Phys<R>& c, const R* nF, bool active, R am, const R* f, R* tau) {
    const R J = det(nF);
    if (D == 2 && c.material == FIXED_COROTATED) {
      const R xx = nF[0] + nF[3], yy = nF[2] - nF[1];
      const R sc = R(1) / dsqrt<R>(xx * xx + yy * yy);
      const R cs = xx * sc, s = yy * sc;
      const R Rm[4] = {cs, -s, s, cs};
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          R acc = 0;
#pragma unroll
          for (int q = 0; q < 2; ++q) acc += (nF[i * 2 + q] - Rm[i * 2 + q]) * nF[j * 2 + q];
          tau[i * D + j] = R(2) * c.mu * acc;
        }
#pragma unroll
      for (int i = 0; i < 2; ++i) tau[i * D + i] += c.la * (J - R(1)) * J;
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          R acc = 0;
#pragma unroll
          for (int q = 0; q < D; ++q) acc += nF[i * D + q] * nF[j * D + q];
          tau[i * D + j] = c.mu * (acc - (i == j ? R(1) : R(0)));
        }
#pragma unroll
      for (int i = 0; i < D; ++i) tau[i * D + i] += c.la * log(J);
    }
    if (active) {
      R u[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        u[i] = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) u[i] += nF[i * D + q] * f[q];
      }
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) tau[i * D + j] += am * u[i] * u[j];
    }
  }

  // d tau / d nF (accumulated into gF); returns d loss / d actuation
  __device__ static R stress_adj(const Phys<R>& c, const R* nF, bool active, R am, const R* f,
                                 const R* gt, R* gF) {
    const R J = det(nF);
    R cf[D * D];
    cof(nF, cf);
    R tr = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) tr += gt[i * D + i];
    if (D == 2 && c.material == FIXED_COROTATED) {
      const R xx = nF[0] + nF[3], yy = nF[2] - nF[1];
      const R r2 = xx * xx + yy * yy, r = dsqrt<R>(r2), r3 = r2 * r;
      const R cs = xx / r, s = yy / r;
      const R Rm[4] = {cs, -s, s, cs};
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          R acc = 0, acc2 = 0;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            acc += (gt[i * 2 + j] + gt[j * 2 + i]) * nF[j * 2 + q];
            acc2 += gt[j * 2 + i] * Rm[j * 2 + q];
          }
          gF[i * 2 + q] += R(2) * c.mu * acc - R(2) * c.mu * acc2;
        }
      R gR[4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          R acc = 0;
#pragma unroll
          for (int j = 0; j < 2; ++j) acc += gt[i * 2 + j] * nF[j * 2 + q];
          gR[i * 2 + q] = R(-2) * c.mu * acc;
        }
      const R gc = gR[0] + gR[3], gs = -gR[1] + gR[2];
      const R gxx = gc * yy * yy / r3 - gs * xx * yy / r3;
      const R gyy = -gc * xx * yy / r3 + gs * xx * xx / r3;
      gF[0] += gxx; gF[3] += gxx; gF[2] += gyy; gF[1] -= gyy;
      const R gJ = c.la * (R(2) * J - R(1)) * tr;
#pragma unroll
      for (int e = 0; e < 4; ++e) gF[e] += gJ * cf[e];
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int q = 0; q < D; ++q) {
          R acc = 0;
#pragma unroll
          for (int j = 0; j < D; ++j) acc += (gt[i * D + j] + gt[j * D + i]) * nF[j * D + q];
          gF[i * D + q] += c.mu * acc;
        }
      const R gJ = c.la * tr / J;
#pragma unroll
      for (int e = 0; e < D * D; ++e) gF[e] += gJ * cf[e];
    }
    R gact = 0;
    if (active) {
      R u[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        u[i] = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) u[i] += nF[i * D + q] * f[q];
      }
      R ga = 0, gu[D];
#pragma unroll
      for (int i = 0; i < D; ++i) gu[i] = 0;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          ga += gt[i * D + j] * u[i] * u[j];
          gu[i] += am * (gt[i * D + j] + gt[j * D + i]) * u[j];
        }
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int q = 0; q < D; ++q) gF[i * D + q] += gu[i] * f[q];
      gact = ga * c.act_strength;
    }
    return gact;
  }

  // product weight of stencil node o and its gradient d w / d fx.  All 3^D
  // stencil nodes lie inside the box of base cells (+2) that the grid
  // kernels visit, so they hold finite values even where a weight is zero.
  __device__ static R wgt(const R w[3][D], const int o[D]) {
    R wt = 1;
#pragma unroll
    for (int d = 0; d < D; ++d) wt *= w[o[d]][d];
    return wt;
  }
  __device__ static void dwgt(const R w[3][D], const R dw[3][D], const int o[D], R dwt[D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      dwt[d] = dw[o[d]][d];
#pragma unroll
      for (int f = 0; f < D; ++f)
        if (f != d) dwt[d] *= w[o[f]][f];
    }
  }
};

// blocked index of node I (per-dim coordinates) of env e
template <typename R, int D>
__device__ __forceinline__ long long node_index(const Phys<R>& c, int e, const int I[D]) {
  constexpr int LOG = Blk<D>::LOG, SIDE = Blk<D>::SIDE;
  long long blk = 0;
  int loc = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    blk = blk * c.nb + (I[d] >> LOG);
    loc = loc * SIDE + (I[d] & (SIDE - 1));
  }
  return ((long long)e * c.nblk + blk) * Blk<D>::NODES + loc;
}

template <typename R>
__device__ __forceinline__ void red4(V4<R>* p, R x, R y, R z, R w);
// 16-byte vector reduction without a return value (PTX red.global.add.v4.f32,
// sm_90+): the issuing thread does not wait for the L2 round trip
template <>
__device__ __forceinline__ void red4<float>(V4<float>* p, float x, float y, float z, float w) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
               :
               : "l"(p), "f"(x), "f"(y), "f"(z), "f"(w)
               : "memory");
}
template <>
__device__ __forceinline__ void red4<double>(V4<double>* p, double x, double y, double z, double w) {
  atomicAdd(&p->x, x);
  atomicAdd(&p->y, y);
  atomicAdd(&p->z, z);
  if (w != 0.0) atomicAdd(&p->w, w);
}

// Runs of consecutive lanes whose particles share a base cell (the
// CLS_MPM_ORDER_BASE_RUNS order puts them next to each other; runs are found
// from the current base cells, so the result is exact for any order).  head:
// first lane of its run; last: the run's last lane; steps: ceil(log2) of the
// warp's longest run.  Invalid lanes are runs of their own.  All lanes call it.
struct WarpRuns {
  int last, steps;
  bool head;
};
template <int D>
__device__ __forceinline__ WarpRuns warp_runs(bool valid, const int base[D]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  bool same = __shfl_up_sync(full, valid ? 1 : 0, 1) != 0 && valid && lane > 0;
#pragma unroll
  for (int d = 0; d < D; ++d) same = (__shfl_up_sync(full, base[d], 1) == base[d]) && same;
  WarpRuns r;
  r.head = !same;
  const unsigned heads = __ballot_sync(full, r.head);
  const unsigned after = lane == 31 ? 0u : (heads >> (lane + 1)) << (lane + 1);
  r.last = after ? __ffs(after) - 2 : 31;
  const int longest = (int)__reduce_max_sync(full, r.head ? (unsigned)(r.last - lane + 1) : 1u);
  r.steps = longest > 1 ? 32 - __clz(longest - 1) : 0;
  return r;
}

// Sum (x, y, z, w) over the lanes of each run (segmented suffix sums by
// shuffles: after the steps, a run's first lane holds the run's total) and
// add the total to *p from that lane, when `issue` is set there.  All lanes
// call it with the same runs.
template <typename R>
__device__ __forceinline__ void run_red4(const WarpRuns& r, V4<R>* p, R x, R y, R z, R w, bool issue) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  for (int s = 0, off = 1; s < r.steps; ++s, off <<= 1) {
    const R ox = __shfl_down_sync(full, x, off), oy = __shfl_down_sync(full, y, off);
    const R oz = __shfl_down_sync(full, z, off), ow = __shfl_down_sync(full, w, off);
    if (lane + off <= r.last) {
      x += ox;
      y += oy;
      z += oz;
      w += ow;
    }
  }
  if (issue && r.head) red4<R>(p, x, y, z, w);
}

// The CTA's box of base cells, extended by the stencil (+2 per dim): the
// nodes a CTA stages in shared memory.  n = 0 when the box exceeds the tile
// capacity (global-atomic fallback).
template <int D>
struct Box {
  int lo[D], ext[D], stride[D], n;
  float rcp[D];
  // tile index of base cell + 0 (add off() of a stencil offset)
  __device__ __forceinline__ int index(const int base[D]) const {
    int li = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) li += (base[d] - lo[d]) * stride[d];
    return li;
  }
  __device__ __forceinline__ int off(const int o[D]) const {
    int li = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) li += o[d] * stride[d];
    return li;
  }
  // node coordinates of tile index li (li < n <= 4096: the float quotient is
  // corrected to the exact one)
  __device__ __forceinline__ void node(int li, int I[D]) const {
#pragma unroll
    for (int d = D - 1; d > 0; --d) {
      int q = (int)(((float)li + 0.5f) * rcp[d]);
      int r = li - q * ext[d];
      if (r < 0) { --q; r += ext[d]; }
      if (r >= ext[d]) { ++q; r -= ext[d]; }
      I[d] = lo[d] + r;
      li = q;
    }
    I[0] = lo[0] + li;
  }
};

// the warp's box (all lanes call it); n = 0 when it exceeds the tile
// capacity or no lane is valid
template <typename R, int D>
__device__ __forceinline__ Box<D> warp_box(const Phys<R>& c, bool valid, const int base[D]) {
  Box<D> bx;
  long long n = 1;
  bool any = true;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int mn = __reduce_min_sync(0xffffffffu, valid ? base[d] : INT_MAX);
    const int mx = __reduce_max_sync(0xffffffffu, valid ? base[d] : INT_MIN);
    any = any && mn <= mx;
    bx.lo[d] = mn;
    bx.ext[d] = any ? mx - mn + 3 : 1;
    bx.rcp[d] = 1.0f / (float)bx.ext[d];
    n *= bx.ext[d];
  }
  int st = 1;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    bx.stride[d] = st;
    st *= bx.ext[d];
  }
  bx.n = (any && c.tile_cap > 0 && n <= c.tile_cap) ? (int)n : 0;
  return bx;
}

// true when two valid lanes of the warp share a base cell (a hash collision
// can only report a shared cell that is not there, which is safe)
template <int D>
__device__ __forceinline__ bool warp_dup_base(bool valid, const int base[D]) {
  unsigned key = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) key = key * 4099u + (unsigned)base[d];
  if (!valid) key = 0xffffffe0u | (threadIdx.x & 31);
  const unsigned mm = __match_any_sync(0xffffffffu, key);
  return __any_sync(0xffffffffu, __popc(mm) > 1);
}

// fold the warp's base cells into the env's box (lane 0: one atomic pair per dim)
template <int D>
__device__ __forceinline__ void warp_bbox(int* bbox, bool valid, const int base[D]) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int mn = __reduce_min_sync(0xffffffffu, valid ? base[d] : INT_MAX);
    const int mx = __reduce_max_sync(0xffffffffu, valid ? base[d] : INT_MIN);
    if ((threadIdx.x & 31) == 0 && mn <= mx) {
      atomicMin(bbox + d, mn);
      atomicMax(bbox + D + d, mx);
    }
  }
}

// stage the grid records under a warp's box into planes [0, NP) of the warp
// tile (component c of node li at tile[c * cap + li]); all lanes call it
template <typename R, int D, int NP>
__device__ __forceinline__ void warp_stage(const Phys<R>& c, const V4<R>* grid, const Box<D>& bx, R* tile,
                                           int cap) {
  for (int li = (int)(threadIdx.x & 31); li < bx.n; li += 32) {
    int I[D];
    bx.node(li, I);
    const V4<R> g = ldg4(grid + node_index<R, D>(c, 0, I));
    tile[li] = g.x;
    if (NP > 1) tile[cap + li] = g.y;
    if (NP > 2) tile[2 * cap + li] = g.z;
    if (NP > 3) tile[3 * cap + li] = g.w;
  }
  __syncwarp();
}

// add v to a warp-tile entry: plain read-modify-write when the warp's lanes
// have distinct base cells (distinct entries per stencil offset), else atomic
template <typename R>
__device__ __forceinline__ void tile_add(R* p, R v, bool atomic) {
  if (atomic) atomicAdd(p, v);
  else *p += v;
}

// warp sum of D values, added to out[0..D) by lane 0
template <typename R, int D>
__device__ __forceinline__ void warp_sum_add(const R v[D], R* out) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    R s = v[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out + d, s);
  }
}

template <typename R>
__device__ __forceinline__ R ld(const R* p) { return __ldg(p); }

// ------------------------------------------------------------------ forward
// G2P of step f (solver_mpm.py:146-165) fused with P2G of step f + 1
// (solver_mpm.py:83-124); either half alone at the ends of a rollout.  The
// 3^D stencil loops are unrolled so that the weights and tile offsets of a
// node are compile-time selections.
template <typename R, int D, int MODE, int SM>
__global__ void __launch_bounds__(kChunk, CLS_MPM_FWD_MIN_BLOCKS) mpm_fwd_kernel(FwdArgs<R> a) {
  using K = Kern<R, D>;
  extern __shared__ __align__(16) unsigned char mpm_smem[];
  const Phys<R>& c = a.c;
  const int cap = c.tile_cap > 0 ? c.tile_cap : 1;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  R* wt_tile = reinterpret_cast<R*>(mpm_smem) + (size_t)wid * kFwdPlanes * cap;  // [kFwdPlanes][cap]
  const int e = blockIdx.x / c.n_chunks, ch = blockIdx.x % c.n_chunks;
  const bool valid = (int)threadIdx.x < c.chunk_len[ch];
  const int p = c.chunk_start[ch] + (valid ? (int)threadIdx.x : 0);
  const long long q = (long long)e * c.P + p;
  const long long EP = c.EP;
  R x[D], v[D], Cm[D * D];
#pragma unroll
  for (int d = 0; d < D; ++d) x[d] = ld(a.x_in + d * EP + q);
  int base[D];
  R fx[D], w[3][D], dw[3][D];

  if (MODE & 1) {
    K::weights(x, c.inv_dx, c.n_grid, base, fx, w, dw);
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = 0;
#pragma unroll
    for (int i = 0; i < D * D; ++i) Cm[i] = 0;
    const V4<R>* gv = a.gv + (size_t)e * c.nblk * Blk<D>::NODES;
    Box<D> gbx;
    gbx.n = 0;
    if (SM & kStageGather) {
      gbx = warp_box<R, D>(c, valid, base);
      if (gbx.n) warp_stage<R, D, D>(c, gv, gbx, wt_tile, cap);
    }
    if (valid) {
      const int li0 = gbx.index(base);
#pragma unroll
      for (int nq = 0; nq < K::NN; ++nq) {
        int o[D];
        K::offs(nq, o);
        const R wt = K::wgt(w, o);
        R g[D];
        if (gbx.n) {
          const int li = li0 + gbx.off(o);
#pragma unroll
          for (int i = 0; i < D; ++i) g[i] = wt_tile[i * cap + li];
        } else {
          int I[D];
#pragma unroll
          for (int d = 0; d < D; ++d) I[d] = base[d] + o[d];
          const V4<R> gg = ldg4(gv + node_index<R, D>(c, 0, I));
          g[0] = gg.x;
          g[1] = gg.y;
          if (D == 3) g[D - 1] = gg.z;
        }
        const R s4 = R(4) * wt * c.inv_dx;
#pragma unroll
        for (int i = 0; i < D; ++i) {
          v[i] += wt * g[i];
#pragma unroll
          for (int j = 0; j < D; ++j) Cm[i * D + j] += s4 * g[i] * ((R)o[j] - fx[j]);
        }
      }
#pragma unroll
      for (int i = 0; i < D; ++i) {
        x[i] += c.dt * v[i];
        a.x_out[i * EP + q] = x[i];
        if (a.v_out) a.v_out[i * EP + q] = v[i];
      }
      if (a.C_out) {
#pragma unroll
        for (int i = 0; i < D * D; ++i) a.C_out[i * EP + q] = Cm[i];
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) v[i] = ld(a.v_in + i * EP + q);
#pragma unroll
    for (int i = 0; i < D * D; ++i) Cm[i] = ld(a.C_in + i * EP + q);
  }
  if (a.csum) {
    R s[D];
    const R pwv = valid ? ld(c.pw + p) : R(0);
#pragma unroll
    for (int d = 0; d < D; ++d) s[d] = pwv * x[d];
    warp_sum_add<R, D>(s, a.csum + (long long)e * D);
  }
  if (!(MODE & 2)) return;

  // P2G of the state (x, v, Cm, F_in)
  K::weights(x, c.inv_dx, c.n_grid, base, fx, w, dw);
  R aff[D * D];  // affine momentum matrix times dx
  {
    R F[D * D], nF[D * D], tau[D * D];
#pragma unroll
    for (int i = 0; i < D * D; ++i) F[i] = ld(a.F_in + i * EP + q);
    K::new_F(Cm, F, c.dt, nF);
    const int m = valid ? ld(c.muscle + p) : -1;
    R f[D];
    R am = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) f[d] = 0;
    if (m >= 0) {
      am = ld(a.act + (long long)e * c.M + m) * c.act_strength;
#pragma unroll
      for (int d = 0; d < D; ++d) f[d] = ld(c.fibre + (long long)d * c.P + p);
    }
    K::stress(c, nF, m >= 0, am, f, tau);
#pragma unroll
    for (int i = 0; i < D * D; ++i) aff[i] = (-c.ks * tau[i] + c.mass * Cm[i]) * c.dx;
    if (a.F_out && valid) {
#pragma unroll
      for (int i = 0; i < D * D; ++i) a.F_out[i * EP + q] = nF[i];
    }
  }
  warp_bbox<D>(a.bbox + (size_t)e * 2 * D, valid, base);
  WarpRuns runs;
  runs.head = true;
  runs.last = lane;
  runs.steps = 0;
  if (c.runs) runs = warp_runs<D>(valid, base);
  Box<D> bx;
  bx.n = 0;
  if (SM & kScatterTile) bx = warp_box<R, D>(c, valid, base);
  const bool dup = bx.n ? warp_dup_base<D>(valid, base) : false;
  if (bx.n) {
    __syncwarp();  // the staged gather is no longer read
    for (int li = lane; li < bx.n; li += 32) {
      wt_tile[li] = 0;
      wt_tile[cap + li] = 0;
      wt_tile[2 * cap + li] = 0;
      wt_tile[3 * cap + li] = 0;
    }
    __syncwarp();
  }
  if (c.runs) {
    // base-cell order: each run of lanes on one base cell adds its 27 node
    // contributions with one reduction per node (run_red4).  The stencil loop
    // is partly rolled: fully unrolled, the shuffles made the kernel
    // instruction-fetch bound (measured slower)
    R mv[D];
#pragma unroll
    for (int i = 0; i < D; ++i) mv[i] = c.mass * v[i];
    // the last axis rolled, the first two unrolled (9 nodes per iteration)
#pragma unroll 1
    for (int ol = 0; ol < (D == 3 ? 3 : 1); ++ol) {
      const R wl = D == 3 ? (ol == 0 ? w[0][D - 1] : (ol == 1 ? w[1][D - 1] : w[2][D - 1])) : R(1);
#pragma unroll
    for (int nq = 0; nq < 9; ++nq) {
      int o[D];
      o[0] = nq % 3;
      o[1] = nq / 3;
      if (D == 3) o[D - 1] = ol;
      const R wt = w[o[0]][0] * w[o[1]][1] * wl;
      R mom[3] = {0, 0, 0};
      long long nidx = 0;
      if (valid) {
#pragma unroll
        for (int i = 0; i < D; ++i) {
          R s = mv[i];
#pragma unroll
          for (int j = 0; j < D; ++j) s += aff[i * D + j] * ((R)o[j] - fx[j]);
          mom[i] = wt * s;
        }
        int I[D];
#pragma unroll
        for (int d = 0; d < D; ++d) I[d] = base[d] + o[d];
        nidx = node_index<R, D>(c, e, I);
      }
      run_red4<R>(runs, a.acc + nidx, mom[0], mom[1], mom[2], valid ? wt * c.mass : R(0), valid);
    }
    }
    return;
  }
  {
    // every lane runs the offsets so that the warp can sync between them
    const int li0 = bx.index(base);
    R mv[D];
#pragma unroll
    for (int i = 0; i < D; ++i) mv[i] = c.mass * v[i];
#pragma unroll
    for (int nq = 0; nq < K::NN; ++nq) {
      int o[D];
      K::offs(nq, o);
      const R wt = K::wgt(w, o);
      if (valid) {
        R mom[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < D; ++i) {
          R s = mv[i];
#pragma unroll
          for (int j = 0; j < D; ++j) s += aff[i * D + j] * ((R)o[j] - fx[j]);
          mom[i] = wt * s;
        }
        if (bx.n) {
          const int li = li0 + bx.off(o);
          tile_add(wt_tile + li, mom[0], dup);
          tile_add(wt_tile + cap + li, mom[1], dup);
          if (D == 3) tile_add(wt_tile + 2 * cap + li, mom[2], dup);
          tile_add(wt_tile + 3 * cap + li, wt * c.mass, dup);
        } else {
          int I[D];
#pragma unroll
          for (int d = 0; d < D; ++d) I[d] = base[d] + o[d];
          red4<R>(a.acc + node_index<R, D>(c, e, I), mom[0], mom[1], mom[2], wt * c.mass);
        }
      }
      if (bx.n) __syncwarp();
    }
  }
  if (bx.n) {
    __syncwarp();
    for (int li = lane; li < bx.n; li += 32) {
      const R m = wt_tile[3 * cap + li];
      if (m == R(0)) continue;  // no particle weight on this node
      int I[D];
      bx.node(li, I);
      red4<R>(a.acc + node_index<R, D>(c, e, I), wt_tile[li], wt_tile[cap + li],
              D == 3 ? wt_tile[2 * cap + li] : R(0), m);
    }
  }
}

// Node n (0 <= n < count) of the blocks under env e's box of base cells
// (+2 per dim); returns false past the last node.
template <typename R, int D>
__device__ __forceinline__ bool box_node(const Phys<R>& c, const int* bb, long long n, int I[D], long long* node) {
  constexpr int LOG = Blk<D>::LOG, SIDE = Blk<D>::SIDE;
  int blo[D], bext[D];
  long long nb = 1;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    if (bb[d] > bb[D + d]) return false;  // no particle
    blo[d] = bb[d] >> LOG;
    bext[d] = ((bb[D + d] + 2) >> LOG) - blo[d] + 1;
    nb *= bext[d];
  }
  if (n >= nb * Blk<D>::NODES) return false;
  long long bi = n / Blk<D>::NODES;
  int loc = (int)(n % Blk<D>::NODES);
  int b[D];
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    b[d] = blo[d] + (int)(bi % bext[d]);
    bi /= bext[d];
  }
  long long blk = 0;
#pragma unroll
  for (int d = 0; d < D; ++d) blk = blk * c.nb + b[d];
  int l = loc;
#pragma unroll
  for (int d = D - 1; d >= 0; --d) {
    I[d] = b[d] * SIDE + (l & (SIDE - 1));
    l >>= LOG;
  }
  *node = blk * Blk<D>::NODES + loc;
  return true;
}

// grid_op (solver_mpm.py:126-144) over the blocks under each env's box:
// velocity, gravity on axis 1, sticky walls.  Consumes (and clears) the
// accumulator, stores (velocity, mass) for G2P and the reverse pass, and
// resets the next step's boxes.  Grid: (x, E).
template <typename R, int D>
__global__ void __launch_bounds__(256) mpm_grid_kernel(Phys<R> c, V4<R>* acc, V4<R>* gv, const int* bbox,
                                                       int* bbox_next) {
  const int e = blockIdx.y;
  int bb[2 * D];
#pragma unroll
  for (int d = 0; d < 2 * D; ++d) bb[d] = bbox[e * 2 * D + d];
  const size_t goff = (size_t)e * c.nblk * Blk<D>::NODES;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;; n += (long long)gridDim.x * blockDim.x) {
    int I[D];
    long long node;
    if (!box_node<R, D>(c, bb, n, I, &node)) break;
    bool wall = false;
#pragma unroll
    for (int d = 0; d < D; ++d) wall |= (I[d] < c.bound || I[d] > c.n_grid - c.bound);
    const V4<R> s = acc[goff + node];
    const R inv_m = R(1) / (s.w + R(1e-10));
    V4<R> o;
    o.x = inv_m * s.x;
    o.y = inv_m * s.y + c.dt * c.gravity;
    o.z = D == 3 ? inv_m * s.z : R(0);
    if (wall) {
      o.x = 0;
      o.y = 0;
      o.z = 0;
    }
    o.w = s.w;
    gv[goff + node] = o;
    acc[goff + node] = V4<R>{0, 0, 0, 0};
  }
  if (bbox_next && blockIdx.x == 0 && threadIdx.x < 2 * D)
    bbox_next[e * 2 * D + threadIdx.x] = threadIdx.x < D ? INT_MAX : INT_MIN;
}

// grid_op^T over the blocks under each env's box: consumes (and clears) the
// velocity adjoint accumulator; writes (d velocity before the update, d mass).
template <typename R, int D>
__global__ void __launch_bounds__(256) mpm_grid_adj_kernel(Phys<R> c, V4<R>* gacc, const V4<R>* gv,
                                                           V4<R>* ga, const int* bbox) {
  const int e = blockIdx.y;
  int bb[2 * D];
#pragma unroll
  for (int d = 0; d < 2 * D; ++d) bb[d] = bbox[e * 2 * D + d];
  const size_t goff = (size_t)e * c.nblk * Blk<D>::NODES;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;; n += (long long)gridDim.x * blockDim.x) {
    int I[D];
    long long node;
    if (!box_node<R, D>(c, bb, n, I, &node)) break;
    bool wall = false;
#pragma unroll
    for (int d = 0; d < D; ++d) wall |= (I[d] < c.bound || I[d] > c.n_grid - c.bound);
    const V4<R> g = gacc[goff + node];
    const V4<R> s = gv[goff + node];
    const R inv_m = R(1) / (s.w + R(1e-10));
    V4<R> o{0, 0, 0, 0};
    if (!wall) {
      // velocity before the update: v - dt g e_1 (momentum / mass)
      const R vy = s.y - c.dt * c.gravity;
      o.x = g.x * inv_m;
      o.y = g.y * inv_m;
      o.z = D == 3 ? g.z * inv_m : R(0);
      o.w = -(g.x * s.x + g.y * vy + (D == 3 ? g.z * s.z : R(0))) * inv_m;
    }
    ga[goff + node] = o;
    gacc[goff + node] = V4<R>{0, 0, 0, 0};
  }
}

// ------------------------------------------------------------------ reverse
// P2G^T of step f + seed of step f (mode bit 1), then G2P^T of step h (mode
// bit 2).  Adjoint of solver_mpm.py:83-124 and :146-165.
template <typename R, int D, int MODE, int SM>
__global__ void __launch_bounds__(kChunk, CLS_MPM_ADJ_MIN_BLOCKS) mpm_adj_kernel(AdjArgs<R> a) {
  using K = Kern<R, D>;
  extern __shared__ __align__(16) unsigned char mpm_smem[];
  const Phys<R>& c = a.c;
  const int cap = c.tile_cap > 0 ? c.tile_cap : 1;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  R* wt_tile = reinterpret_cast<R*>(mpm_smem) + (size_t)wid * kAdjPlanes * cap;  // [kAdjPlanes][cap]
  const int e = blockIdx.x / c.n_chunks, ch = blockIdx.x % c.n_chunks;
  const bool valid = (int)threadIdx.x < c.chunk_len[ch];
  const int p = c.chunk_start[ch] + (valid ? (int)threadIdx.x : 0);
  const long long q = (long long)e * c.P + p;
  const long long EP = c.EP;
  const size_t goff = (size_t)e * c.nblk * Blk<D>::NODES;
  int base[D];
  R fx[D], w[3][D], dw[3][D];
  R ax[D], av[D], aC[D * D];

  if (MODE & 1) {
    R x[D], vp[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
      x[d] = ld(a.x_f + d * EP + q);
      vp[d] = ld(a.v_f + d * EP + q);
    }
    K::weights(x, c.inv_dx, c.n_grid, base, fx, w, dw);
    const int m = valid ? ld(c.muscle + p) : -1;
    R f[D], am = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) f[d] = 0;
    if (m >= 0) {
      am = ld(a.act_f + (long long)e * c.M + m) * c.act_strength;
#pragma unroll
      for (int d = 0; d < D; ++d) f[d] = ld(c.fibre + (long long)d * c.P + p);
    }
    R aff[D * D];  // affine momentum matrix times dx
    {
      R Cp[D * D], Fp[D * D], nF[D * D], tau[D * D];
#pragma unroll
      for (int i = 0; i < D * D; ++i) {
        Cp[i] = ld(a.C_f + i * EP + q);
        Fp[i] = ld(a.F_f + i * EP + q);
      }
      K::new_F(Cp, Fp, c.dt, nF);
      K::stress(c, nF, m >= 0, am, f, tau);
#pragma unroll
      for (int i = 0; i < D * D; ++i) aff[i] = (-c.ks * tau[i] + c.mass * Cp[i]) * c.dx;
    }
    R gaff[D * D], gfx[D];  // gaff: d loss / d (affine matrix times dx)
#pragma unroll
    for (int i = 0; i < D * D; ++i) gaff[i] = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
      gfx[i] = 0;
      av[i] = 0;
    }
    Box<D> gbx;
    gbx.n = 0;
    if (SM & kStageGather) {
      gbx = warp_box<R, D>(c, valid, base);
      if (gbx.n) warp_stage<R, D, 4>(c, a.ga + goff, gbx, wt_tile, cap);
    }
    if (valid) {
      const int li0 = gbx.index(base);
#pragma unroll
      for (int nq = 0; nq < K::NN; ++nq) {
        int o[D];
        K::offs(nq, o);
        const R wt = K::wgt(w, o);
        R dwt[D], dp[D], gg[D], ggm;
        K::dwgt(w, dw, o, dwt);
#pragma unroll
        for (int d = 0; d < D; ++d) dp[d] = (R)o[d] - fx[d];
        if (gbx.n) {
          const int li = li0 + gbx.off(o);
#pragma unroll
          for (int i = 0; i < D; ++i) gg[i] = wt_tile[i * cap + li];
          ggm = wt_tile[3 * cap + li];
        } else {
          int I[D];
#pragma unroll
          for (int d = 0; d < D; ++d) I[d] = base[d] + o[d];
          const V4<R> g4 = ldg4(a.ga + goff + node_index<R, D>(c, 0, I));
          gg[0] = g4.x;
          gg[1] = g4.y;
          if (D == 3) gg[D - 1] = g4.z;
          ggm = g4.w;
        }
        R gw = ggm * c.mass;
#pragma unroll
        for (int i = 0; i < D; ++i) {
          R mom = c.mass * vp[i];
#pragma unroll
          for (int j = 0; j < D; ++j) mom += aff[i * D + j] * dp[j];
          gw += gg[i] * mom;
          av[i] += wt * c.mass * gg[i];
          const R wg = wt * gg[i];
#pragma unroll
          for (int j = 0; j < D; ++j) gaff[i * D + j] += wg * dp[j];
        }
#pragma unroll
        for (int j = 0; j < D; ++j) {
          R acc = 0;
#pragma unroll
          for (int i = 0; i < D; ++i) acc += aff[i * D + j] * gg[i];
          gfx[j] -= wt * acc;
        }
#pragma unroll
        for (int d = 0; d < D; ++d) gfx[d] += gw * dwt[d];
      }
    }
    // stress adjoint: reload C, F (cheaper than keeping them live)
    R Cp[D * D], Fp[D * D], gnF[D * D], gact;
    {
      R nF[D * D], gtau[D * D];
#pragma unroll
      for (int i = 0; i < D * D; ++i) {
        Cp[i] = ld(a.C_f + i * EP + q);
        Fp[i] = ld(a.F_f + i * EP + q);
        gtau[i] = -c.ks * c.dx * gaff[i];
        gnF[i] = valid ? ld(a.aF_in + i * EP + q) : R(0);
      }
      K::new_F(Cp, Fp, c.dt, nF);
      gact = K::stress_adj(c, nF, m >= 0, am, f, gtau, gnF);
    }
    // d actuation: warp-aggregated when the warp's particles share a muscle
    {
      const unsigned full = 0xffffffffu;
      const int m0 = __shfl_sync(full, m, 0);
      R* ga_e = a.gact + (long long)e * c.M;
      if (__all_sync(full, m == m0)) {
        R s = gact;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(full, s, o);
        if (lane == 0 && m0 >= 0) atomicAdd(ga_e + m0, s);
      } else if (m >= 0) {
        atomicAdd(ga_e + m, gact);
      }
    }
    // complete the state-f adjoint (+ loss seed of step f)
#pragma unroll
    for (int d = 0; d < D; ++d) {
      R s = 0;
      if (a.seed_w != R(0) && valid)
        s = R(2) * a.seed_w * (ld(a.csum + (long long)e * D + d) / a.pw_sum - ld(a.target + (long long)e * D + d)) *
            ld(c.pw + p) / a.pw_sum;
      ax[d] = (valid ? ld(a.ax_in + d * EP + q) : R(0)) + gfx[d] * c.inv_dx + s;
    }
    R* aF_dst = (MODE & 2) ? a.aF_out : a.out_aF;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R accC = 0, accF = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
          accC += gnF[i * D + k] * Fp[j * D + k];
          accF += ((k == i ? R(1) : R(0)) + c.dt * Cp[k * D + i]) * gnF[k * D + j];
        }
        aC[i * D + j] = c.mass * c.dx * gaff[i * D + j] + c.dt * accC;
        if (valid) aF_dst[(i * D + j) * EP + q] = accF;
      }
    if (!(MODE & 2)) {
      if (valid) {
#pragma unroll
        for (int d = 0; d < D; ++d) {
          a.out_ax[d * EP + q] = ax[d];
          a.out_av[d * EP + q] = av[d];
        }
#pragma unroll
        for (int i = 0; i < D * D; ++i) a.out_aC[i * EP + q] = aC[i];
      }
      return;
    }
  } else {
    // first reverse step: a_x(T) is the loss seed of step T, a_v = a_C = 0
#pragma unroll
    for (int d = 0; d < D; ++d) {
      ax[d] = 0;
      av[d] = 0;
      if (a.seed_w != R(0) && valid)
        ax[d] = R(2) * a.seed_w * (ld(a.csum + (long long)e * D + d) / a.pw_sum - ld(a.target + (long long)e * D + d)) *
                ld(c.pw + p) / a.pw_sum;
    }
#pragma unroll
    for (int i = 0; i < D * D; ++i) aC[i] = 0;
    if (valid) {
#pragma unroll
      for (int i = 0; i < D * D; ++i) a.aF_out[i * EP + q] = 0;
    }
  }

  // G2P^T of step h: gather the grid velocity of step h through L1, scatter
  // the velocity adjoint through the warp tile
  R xh[D];
#pragma unroll
  for (int d = 0; d < D; ++d) xh[d] = ld(a.x_h + d * EP + q);
  K::weights(xh, c.inv_dx, c.n_grid, base, fx, w, dw);
  // planes 0..2: the staged grid velocity; planes 3..5: the scatter tile
  Box<D> bx;
  bx.n = 0;
  if (SM & (kStageGather | kScatterTile)) bx = warp_box<R, D>(c, valid, base);
  const bool stage = (SM & kStageGather) && bx.n;
  const bool tile = (SM & kScatterTile) && bx.n;
  const bool dup = tile ? warp_dup_base<D>(valid, base) : false;
  if (bx.n) {
    __syncwarp();  // the P2G^T staging is no longer read
    if (stage) warp_stage<R, D, D>(c, a.gv_h + goff, bx, wt_tile, cap);
    if (tile) {
      for (int li = lane; li < bx.n; li += 32) {
        wt_tile[3 * cap + li] = 0;
        wt_tile[4 * cap + li] = 0;
        wt_tile[5 * cap + li] = 0;
      }
      __syncwarp();
    }
  }
  {
    R gvt[D], gfx[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      gvt[i] = av[i] + c.dt * ax[i];
      gfx[i] = 0;
    }
    const R s4 = R(4) * c.inv_dx;
    const int li0 = bx.index(base);
#pragma unroll
    for (int nq = 0; nq < K::NN; ++nq) {
      int o[D];
      K::offs(nq, o);
      const R wt = K::wgt(w, o);
      if (valid) {
        R dwt[D], dp[D], g[D];
        K::dwgt(w, dw, o, dwt);
        int I[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          dp[d] = (R)o[d] - fx[d];
          I[d] = base[d] + o[d];
        }
        const long long gidx = node_index<R, D>(c, e, I);
        const int li = li0 + bx.off(o);
        if (stage) {
#pragma unroll
          for (int i = 0; i < D; ++i) g[i] = wt_tile[i * cap + li];
        } else {
          const V4<R> g4 = ldg4(a.gv_h + gidx);
          g[0] = g4.x;
          g[1] = g4.y;
          if (D == 3) g[D - 1] = g4.z;
        }
        R gw = 0, sc[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < D; ++i) {
          R gGC = 0;
#pragma unroll
          for (int j = 0; j < D; ++j) gGC += aC[i * D + j] * dp[j];
          sc[i] = wt * (gvt[i] + s4 * gGC);
          gw += g[i] * (gvt[i] + s4 * gGC);
        }
#pragma unroll
        for (int j = 0; j < D; ++j) {
          R acc = 0;
#pragma unroll
          for (int i = 0; i < D; ++i) acc += aC[i * D + j] * g[i];
          gfx[j] -= s4 * wt * acc;
        }
#pragma unroll
        for (int d = 0; d < D; ++d) gfx[d] += gw * dwt[d];
        if (tile) {
          tile_add(wt_tile + 3 * cap + li, sc[0], dup);
          tile_add(wt_tile + 4 * cap + li, sc[1], dup);
          if (D == 3) tile_add(wt_tile + 5 * cap + li, sc[2], dup);
        } else {
          red4<R>(a.gacc + gidx, sc[0], sc[1], sc[2], R(0));
        }
      }
      if (tile) __syncwarp();
    }
    if (valid) {
#pragma unroll
      for (int d = 0; d < D; ++d) a.ax_out[d * EP + q] = ax[d] + gfx[d] * c.inv_dx;
    }
  }
  if (tile) {
    __syncwarp();
    for (int li = lane; li < bx.n; li += 32) {
      const R s0 = wt_tile[3 * cap + li], s1 = wt_tile[4 * cap + li], s2 = D == 3 ? wt_tile[5 * cap + li] : R(0);
      if (s0 == R(0) && s1 == R(0) && s2 == R(0)) continue;
      int I[D];
      bx.node(li, I);
      red4<R>(a.gacc + node_index<R, D>(c, e, I), s0, s1, s2, R(0));
    }
  }
}

// empty boxes (min = INT_MAX, max = INT_MIN) for n_env envs
template <int D>
__global__ void mpm_bbox_reset_kernel(int* bbox, int n_env) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_env * 2 * D) bbox[i] = (i % (2 * D)) < D ? INT_MAX : INT_MIN;
}

}  // namespace mpm
}  // namespace cls
