// mpm_runtime.cu -- cls_mpm_* C ABI: MLS-MPM episodes with checkpointed
// reverse passes.  The first pass keeps the particle state every K steps; the
// reverse pass recomputes each segment's states and grids into a record (two
// records, alternating by segment), then runs one grid-adjoint and one fused
// particle-adjoint launch per step.  The reference's advance_core_grad
// (solver_mpm.py:182-190) rebuilds a step's grid before its adjoint; here the
// grid recorded by the recompute is reused.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/cls_b200.h"
#include "cls_profile.cuh"
#include "mpm_kernels.cuh"

namespace cls {
namespace mpm {

static thread_local std::string g_mpm_create_error;

struct MFail {
  int code;
  std::string msg;
};

#define MPM_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw MFail{e_ == cudaErrorMemoryAllocation ? CLS_ERR_OOM : CLS_ERR_CUDA,          \
                  std::string(#call) + ": " + cudaGetErrorString(e_)};                   \
  } while (0)
#define MPM_REQUIRE(cond, msg)                                                           \
  do {                                                                                   \
    if (!(cond)) throw MFail{CLS_ERR_INVALID, (msg)};                                    \
  } while (0)

template <typename T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t c) {
    if (p) cudaFree(p);
    p = nullptr;
    n = c;
    if (c) MPM_CUDA(cudaMalloc(&p, sizeof(T) * c));
  }
  ~Buf() { if (p) cudaFree(p); }
};

class MpmBase {
 public:
  virtual ~MpmBase() = default;
  std::string err;
  cudaStream_t stream = nullptr;
  virtual void set_state(const double* x0, const double* v0) = 0;
  virtual void set_actuation(const double* act) = 0;
  virtual void set_loss(const double* w, const double* target, const double* pw) = 0;
  virtual void forward(int steps) = 0;
  virtual double loss() = 0;
  virtual void backward() = 0;
  virtual void final_state(double* x, double* v, double* C, double* F) = 0;
  virtual void grads(double* gact, double* gx0, double* gv0, double* gC0, double* gF0) = 0;
  virtual void centers(double* c) = 0;
  virtual void graph_capture(int steps) = 0;
  virtual void graph_launch() = 0;
  virtual void profile_enable(bool on) = 0;
  virtual void profile_read(double* ms, long long* launches, bool reset) = 0;
};

// launch categories of the per-kernel profile (CLS_MPM_PROFILE_KINDS)
enum MpmKind : int { MK_PFWD = 0, MK_PREC, MK_GRID, MK_PADJ, MK_GADJ, MK_OTHER, MK_COUNT };

template <typename R, int D>
class MpmImpl final : public MpmBase {
  using V = V4<R>;

 public:
  MpmImpl(const cls_mpm_body& b, const cls_mpm_params& p, int n_envs) : p_(p) {
    E_ = n_envs;
    P_ = b.n_particles;
    M_ = std::max(1, b.n_muscles);
    T_ = p.max_steps;
    K_ = std::max(1, p.checkpoint_every);
    n_grid_ = p.n_grid;
    MPM_REQUIRE(M_ <= kMaxMuscles, "at most 256 muscle groups");
    MPM_REQUIRE(E_ <= 65535, "at most 65535 envs per handle");
    MPM_REQUIRE((long long)E_ * P_ < (1LL << 31) / (D * D), "too many particles");
    // warp tiles (staged gathers and scatter tiles) only with tile_nodes > 0:
    // both measured slower than L1 gathers and direct vector reductions
    MPM_REQUIRE(p.tile_nodes <= 1024, "tile_nodes must be at most 1024");
    sm_mode_ = p.tile_nodes > 0 ? (kStageGather | kScatterTile) : 0;
    tile_cap_ = p.tile_nodes > 0 ? p.tile_nodes : 0;
    MPM_REQUIRE(p.particle_order == CLS_MPM_ORDER_CELLS || p.particle_order == CLS_MPM_ORDER_BASE_RUNS,
                "particle_order must be CLS_MPM_ORDER_CELLS or CLS_MPM_ORDER_BASE_RUNS");
    MPM_REQUIRE(p.particle_order == CLS_MPM_ORDER_CELLS || tile_cap_ == 0,
                "CLS_MPM_ORDER_BASE_RUNS needs tile_nodes <= 0");
    runs_ = p.particle_order == CLS_MPM_ORDER_BASE_RUNS;
    nb_ = (n_grid_ + Blk<D>::SIDE - 1) / Blk<D>::SIDE;
    nblk_ = 1;
    for (int d = 0; d < D; ++d) nblk_ *= nb_;
    MPM_REQUIRE((long long)E_ * nblk_ < (1LL << 31), "grid too large");
    slots_ = std::max(K_, 2);
    n_ckpt_ = (T_ + K_ - 1) / K_ + 1;
    build_order(b);
    n_chunks_ = (int)chunk_start_h_.size();
    MPM_REQUIRE((long long)E_ * n_chunks_ < (1LL << 31), "too many particle chunks");

    const size_t EP = (size_t)E_ * P_, VX = EP * D, VM = EP * D * D;
    const size_t nodes = (size_t)E_ * nblk_ * Blk<D>::NODES;
    ck_x_.alloc(n_ckpt_ * VX); ck_v_.alloc(n_ckpt_ * VX);
    ck_C_.alloc(n_ckpt_ * VM); ck_F_.alloc(n_ckpt_ * VM);
    for (int s = 0; s < 2; ++s) {
      X_[s].alloc(VX); Fw_[s].alloc(VM);
      RX_[s].alloc(K_ * VX); RV_[s].alloc(K_ * VX); RC_[s].alloc(K_ * VM); RF_[s].alloc(K_ * VM);
      AX_[s].alloc(VX); AF_[s].alloc(VM);
      gv_[s].alloc(slots_ * nodes);
    }
    bboxes_.alloc((size_t)2 * slots_ * E_ * 2 * D);
    acc_.alloc(nodes); gacc_.alloc(nodes); ga_.alloc(nodes);
    fin_x_.alloc(VX); fin_v_.alloc(VX); fin_C_.alloc(VM); fin_F_.alloc(VM);
    out_ax_.alloc(VX); out_av_.alloc(VX); out_aC_.alloc(VM); out_aF_.alloc(VM);
    act_.alloc((size_t)T_ * E_ * M_); gact_.alloc((size_t)T_ * E_ * M_);
    csum_.alloc((size_t)(T_ + 1) * E_ * D);
    target_.alloc((size_t)(T_ + 1) * E_ * D);
    muscle_.alloc(P_); fibre_.alloc((size_t)P_ * D); pw_.alloc(P_);
    chunk_start_.alloc(n_chunks_); chunk_len_.alloc(n_chunks_);
    MPM_CUDA(cudaMemcpy(chunk_start_.p, chunk_start_h_.data(), sizeof(int) * n_chunks_, cudaMemcpyHostToDevice));
    MPM_CUDA(cudaMemcpy(chunk_len_.p, chunk_len_h_.data(), sizeof(int) * n_chunks_, cudaMemcpyHostToDevice));
    // accumulators and flags start (and stay, between steps) zero; the grid
    // buffers start zero so that unvisited nodes hold finite values
    MPM_CUDA(cudaMemset(acc_.p, 0, sizeof(V) * nodes));
    MPM_CUDA(cudaMemset(gacc_.p, 0, sizeof(V) * nodes));
    MPM_CUDA(cudaMemset(ga_.p, 0, sizeof(V) * nodes));
    for (int s = 0; s < 2; ++s) MPM_CUDA(cudaMemset(gv_[s].p, 0, sizeof(V) * slots_ * nodes));

    std::vector<int> mus(P_, -1);
    for (int i = 0; i < P_; ++i) {
      const int m = b.muscle ? b.muscle[perm_[i]] : -1;
      MPM_REQUIRE(m >= -1 && m < M_, "muscle index out of range");
      mus[i] = m;
    }
    MPM_CUDA(cudaMemcpy(muscle_.p, mus.data(), sizeof(int) * P_, cudaMemcpyHostToDevice));
    std::vector<R> fib((size_t)P_ * D, R(0));
    for (int i = 0; i < P_; ++i)
      for (int d = 0; d < D; ++d)
        fib[(size_t)d * P_ + i] = b.fibre ? (R)b.fibre[(size_t)perm_[i] * D + d] : (d == 1 ? R(1) : R(0));
    MPM_CUDA(cudaMemcpy(fibre_.p, fib.data(), sizeof(R) * fib.size(), cudaMemcpyHostToDevice));
    std::vector<R> pw(P_, R(1));
    pw_sum_ = P_;
    MPM_CUDA(cudaMemcpy(pw_.p, pw.data(), sizeof(R) * P_, cudaMemcpyHostToDevice));
    loss_w_.assign(T_ + 1, 0.0);
    MPM_CUDA(cudaMemset(act_.p, 0, sizeof(R) * act_.n));
    MPM_CUDA(cudaMemset(target_.p, 0, sizeof(R) * target_.n));
    // shared-memory opt-in for the tile
    fwd_smem_ = tile_cap_ > 0 ? (size_t)kWarps * kFwdPlanes * tile_cap_ * sizeof(R) : 0;
    adj_smem_ = tile_cap_ > 0 ? (size_t)kWarps * kAdjPlanes * tile_cap_ * sizeof(R) : 0;
    set_smem_attrs<kStageGather | kScatterTile>();
    // initial state: body positions in every env, v = C = 0, F = I
    std::vector<double> x0(EP * D), v0(EP * D, 0.0);
    for (int e = 0; e < E_; ++e)
      std::memcpy(&x0[(size_t)e * P_ * D], b.positions, sizeof(double) * P_ * D);
    set_state(x0.data(), v0.data());
    MPM_CUDA(cudaDeviceSynchronize());
  }

  ~MpmImpl() override {
    if (gexec_) cudaGraphExecDestroy(gexec_);
    if (graph_) cudaGraphDestroy(graph_);
  }

  // Internal particle order: Morton order of the initial cells (ties by
  // position), cut into chunks of at most kChunk (below); inside a chunk the
  // i-th particle of every cell comes first, so that a warp's lanes sit in
  // different cells.
  // CLS_MPM_ORDER_BASE_RUNS: the same Morton order over the stencils' base
  // cells (floor(x / dx - 0.5)), cut into plain runs of kChunk, without the
  // interleave, so that particles sharing a base cell sit in consecutive lanes.
  void build_order(const cls_mpm_body& b) {
    std::vector<unsigned long long> key(P_);
    std::map<unsigned long long, int> cells;
    const double shift = runs_ ? 0.5 : 0.0;
    for (int u = 0; u < P_; ++u) {
      unsigned long long k = 0;
      int cc[D];
      for (int d = 0; d < D; ++d) {
        const double c = std::floor(b.positions[(size_t)u * D + d] * n_grid_ - shift);
        cc[d] = (int)std::min<double>(std::max<double>(c, 0.0), n_grid_ - 1);
      }
      for (int bit = 20; bit >= 0; --bit)
        for (int d = 0; d < D; ++d) k = (k << 1) | ((cc[d] >> bit) & 1);
      key[u] = k;
      cells[k] += 1;
    }
    std::vector<int> order(P_);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
      if (key[a] != key[c]) return key[a] < key[c];
      for (int d = 0; d < D; ++d) {
        const double pa = b.positions[(size_t)a * D + d], pc = b.positions[(size_t)c * D + d];
        if (pa != pc) return pa < pc;
      }
      return false;
    });
    const int per_cell = std::max(1, std::min(8, (int)std::lround((double)P_ / (double)cells.size())));
    // chunks of at most kChunk particles; with the interleave below, the
    // warps of a full chunk each hold particles of distinct cells.  Default:
    // plain runs in Morton order (every thread of a CTA busy); with
    // CLS_MPM_CHUNK_GROUPS a chunk stays inside one aligned Morton group of 32
    // (3D) or 64 (2D) cells (compact boxes for the shared-memory tiles, but
    // about 60 % of the threads busy on a voxelised body)
#ifndef CLS_MPM_CHUNK_GROUPS
#define CLS_MPM_CHUNK_GROUPS 0
#endif
    const bool grouped = CLS_MPM_CHUNK_GROUPS != 0;
    const int group_shift = D == 3 ? 5 : 6;
    chunk_start_h_.clear();
    chunk_len_h_.clear();
    for (int i = 0; i < P_;) {
      const unsigned long long g = key[order[i]] >> group_shift;
      int j = i;
      while (j < P_ && j - i < kChunk && (!grouped || (key[order[j]] >> group_shift) == g)) ++j;
      chunk_start_h_.push_back(i);
      chunk_len_h_.push_back(j - i);
      i = j;
    }
    perm_.resize(P_);
    for (size_t ch = 0; ch < chunk_start_h_.size(); ++ch) {
      const int c0 = chunk_start_h_[ch], len = chunk_len_h_[ch];
      std::vector<int> pos(len);
      std::iota(pos.begin(), pos.end(), 0);
      if (!runs_)
        std::stable_sort(pos.begin(), pos.end(), [&](int a, int c) { return a % per_cell < c % per_cell; });
      for (int t = 0; t < len; ++t) perm_[c0 + t] = order[c0 + pos[t]];
    }
  }

  Phys<R> phys() const {
    Phys<R> c;
    std::memset(&c, 0, sizeof(c));
    c.E = E_; c.P = P_; c.M = M_; c.material = p_.material; c.n_chunks = n_chunks_; c.tile_cap = tile_cap_;
    c.runs = runs_ ? 1 : 0;
    c.n_grid = n_grid_; c.nb = nb_; c.bound = p_.bound; c.nblk = nblk_; c.EP = (long long)E_ * P_;
    c.dx = (R)(1.0 / n_grid_); c.inv_dx = (R)n_grid_; c.dt = (R)p_.dt;
    c.ks = (R)(p_.dt * p_.p_vol * 4.0 * n_grid_ * n_grid_);
    c.mu = (R)p_.mu; c.la = (R)p_.la; c.act_strength = (R)p_.act_strength;
    c.gravity = (R)p_.gravity; c.mass = (R)p_.mass;
    c.muscle = muscle_.p; c.fibre = fibre_.p; c.pw = pw_.p;
    c.chunk_start = chunk_start_.p; c.chunk_len = chunk_len_.p;
    return c;
  }

  size_t VX() const { return (size_t)E_ * P_ * D; }
  size_t VM() const { return (size_t)E_ * P_ * D * D; }
  size_t NODES() const { return (size_t)E_ * nblk_ * Blk<D>::NODES; }

  // checkpoint s, record slot k of record r, work buffers
  R* ckx(int s) { return ck_x_.p + (size_t)s * VX(); }
  R* ckv(int s) { return ck_v_.p + (size_t)s * VX(); }
  R* ckC(int s) { return ck_C_.p + (size_t)s * VM(); }
  R* ckF(int s) { return ck_F_.p + (size_t)s * VM(); }
  V* gv(int r, int k) { return gv_[r].p + (size_t)k * NODES(); }
  int* bbox(int r, int k) { return bboxes_.p + ((size_t)r * slots_ + k) * E_ * 2 * D; }
  // state of step t0(s) + k of segment s (slot 0 is the checkpoint)
  R* rx(int s, int k) { return k == 0 ? ckx(s) : RX_[s % 2].p + (size_t)k * VX(); }
  R* rv(int s, int k) { return k == 0 ? ckv(s) : RV_[s % 2].p + (size_t)k * VX(); }
  R* rC(int s, int k) { return k == 0 ? ckC(s) : RC_[s % 2].p + (size_t)k * VM(); }
  R* rF(int s, int k) { return k == 0 ? ckF(s) : RF_[s % 2].p + (size_t)k * VM(); }
  // first pass: x and F of step g (checkpoint steps live in the checkpoints)
  R* fx(int g) { return g % K_ == 0 ? ckx(g / K_) : X_[g % 2].p; }
  R* fF(int g) { return g % K_ == 0 ? ckF(g / K_) : Fw_[g % 2].p; }
  const R* act(int g) const { return act_.p + (size_t)g * E_ * M_; }

  int particle_grid() const { return E_ * n_chunks_; }

  template <typename F>
  void timed(int kind, F&& f) {
    MPM_CUDA(prof_.run(kind, stream, std::forward<F>(f)));
  }

  template <int SM>
  void set_smem_attrs() {
    MPM_CUDA(cudaFuncSetAttribute(mpm_fwd_kernel<R, D, 1, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem_));
    MPM_CUDA(cudaFuncSetAttribute(mpm_fwd_kernel<R, D, 2, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem_));
    MPM_CUDA(cudaFuncSetAttribute(mpm_fwd_kernel<R, D, 3, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem_));
    MPM_CUDA(cudaFuncSetAttribute(mpm_adj_kernel<R, D, 1, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adj_smem_));
    MPM_CUDA(cudaFuncSetAttribute(mpm_adj_kernel<R, D, 2, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adj_smem_));
    MPM_CUDA(cudaFuncSetAttribute(mpm_adj_kernel<R, D, 3, SM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adj_smem_));
  }
  template <int SM>
  void fwd_t(int mode, const FwdArgs<R>& a) {
    if (mode == 1) mpm_fwd_kernel<R, D, 1, SM><<<particle_grid(), kChunk, fwd_smem_, stream>>>(a);
    else if (mode == 2) mpm_fwd_kernel<R, D, 2, SM><<<particle_grid(), kChunk, fwd_smem_, stream>>>(a);
    else mpm_fwd_kernel<R, D, 3, SM><<<particle_grid(), kChunk, fwd_smem_, stream>>>(a);
  }
  template <int SM>
  void adj_t(int mode, const AdjArgs<R>& a) {
    if (mode == 1) mpm_adj_kernel<R, D, 1, SM><<<particle_grid(), kChunk, adj_smem_, stream>>>(a);
    else if (mode == 2) mpm_adj_kernel<R, D, 2, SM><<<particle_grid(), kChunk, adj_smem_, stream>>>(a);
    else mpm_adj_kernel<R, D, 3, SM><<<particle_grid(), kChunk, adj_smem_, stream>>>(a);
  }
  void launch_fwd(int mode, const FwdArgs<R>& a, int kind) {
    timed(kind, [&] {
      if (sm_mode_ == 0) fwd_t<0>(mode, a);
      else fwd_t<kStageGather | kScatterTile>(mode, a);
    });
  }
  void launch_adj(int mode, const AdjArgs<R>& a) {
    timed(MK_PADJ, [&] {
      if (sm_mode_ == 0) adj_t<0>(mode, a);
      else adj_t<kStageGather | kScatterTile>(mode, a);
    });
  }
  dim3 grid_dims() const { return dim3((unsigned)std::max(1, 148 * 4 / E_), (unsigned)E_); }
  void launch_grid(V* gvo, int r, int k, int* bbox_next) {
    const Phys<R> c = phys();
    timed(MK_GRID, [&] {
      mpm_grid_kernel<R, D><<<grid_dims(), 256, 0, stream>>>(c, acc_.p, gvo, bbox(r, k), bbox_next);
    });
  }
  void reset_bbox(int r, int k) {
    timed(MK_OTHER, [&] {
      mpm_bbox_reset_kernel<D><<<(E_ * 2 * D + 255) / 256, 256, 0, stream>>>(bbox(r, k), E_);
    });
  }

  FwdArgs<R> fwd_args() const {
    FwdArgs<R> a;
    std::memset(&a, 0, sizeof(a));
    a.c = phys();
    a.acc = acc_.p;
    return a;
  }

  // ---------------------------------------------------------------- forward
  void forward(int steps) override {
    MPM_REQUIRE(steps >= 1 && steps <= T_, "steps must be in [1, max_steps]");
    steps_ = steps;
    const size_t cslab = (size_t)E_ * D;
    timed(MK_OTHER, [&] { cudaMemsetAsync(csum_.p, 0, sizeof(R) * (steps + 1) * cslab, stream); });
    reset_bbox(0, 0);
    {  // P2G of step 0
      FwdArgs<R> a = fwd_args();
      a.x_in = ckx(0); a.v_in = ckv(0); a.C_in = ckC(0); a.F_in = ckF(0);
      a.F_out = steps > 1 ? fF(1) : fin_F_.p;
      a.act = act(0);
      a.bbox = bbox(0, 0);
      a.csum = csum_.p;
      launch_fwd(2, a, MK_PFWD);
    }
    launch_grid(gv(0, 0), 0, 0, steps > 1 ? bbox(0, 1) : nullptr);
    for (int f = 0; f + 1 < steps; ++f) {
      const int g = f + 1;
      FwdArgs<R> a = fwd_args();
      a.x_in = fx(f);
      a.gv = gv(0, f % 2);
      a.x_out = fx(g);
      if (g % K_ == 0) { a.v_out = ckv(g / K_); a.C_out = ckC(g / K_); }
      a.F_in = fF(g);
      a.F_out = g + 1 <= steps - 1 ? fF(g + 1) : fin_F_.p;
      a.act = act(g);
      a.bbox = bbox(0, g % 2);
      a.csum = csum_.p + (size_t)g * cslab;
      launch_fwd(3, a, MK_PFWD);
      launch_grid(gv(0, g % 2), 0, g % 2, g + 1 <= steps - 1 ? bbox(0, f % 2) : nullptr);
    }
    {  // G2P of the last step
      FwdArgs<R> a = fwd_args();
      a.x_in = fx(steps - 1);
      a.gv = gv(0, (steps - 1) % 2);
      a.x_out = fin_x_.p; a.v_out = fin_v_.p; a.C_out = fin_C_.p;
      a.csum = csum_.p + (size_t)steps * cslab;
      launch_fwd(1, a, MK_PFWD);
    }
    MPM_CUDA(cudaGetLastError());
    fwd_done_ = true;
    bwd_done_ = false;
  }

  // states and grids of segment s recomputed into its record (record s % 2)
  void recompute(int s) {
    const int r = s % 2, t0 = s * K_, len = std::min(K_, steps_ - t0);
    reset_bbox(r, 0);
    {
      FwdArgs<R> a = fwd_args();
      a.x_in = rx(s, 0); a.v_in = rv(s, 0); a.C_in = rC(s, 0); a.F_in = rF(s, 0);
      a.F_out = len > 1 ? rF(s, 1) : nullptr;
      a.act = act(t0);
      a.bbox = bbox(r, 0);
      launch_fwd(2, a, MK_PREC);
    }
    launch_grid(gv(r, 0), r, 0, len > 1 ? bbox(r, 1) : nullptr);
    for (int k = 0; k + 1 < len; ++k) {
      FwdArgs<R> a = fwd_args();
      a.x_in = rx(s, k);
      a.gv = gv(r, k);
      a.x_out = rx(s, k + 1); a.v_out = rv(s, k + 1); a.C_out = rC(s, k + 1);
      a.F_in = rF(s, k + 1);
      a.F_out = k + 2 < len ? rF(s, k + 2) : nullptr;
      a.act = act(t0 + k + 1);
      a.bbox = bbox(r, k + 1);
      launch_fwd(3, a, MK_PREC);
      launch_grid(gv(r, k + 1), r, k + 1, k + 2 < len ? bbox(r, k + 2) : nullptr);
    }
  }

  double loss() override {
    MPM_REQUIRE(fwd_done_, "cls_mpm_loss before a forward rollout");
    std::vector<R> c((size_t)(steps_ + 1) * E_ * D), tg((size_t)(steps_ + 1) * E_ * D);
    MPM_CUDA(cudaMemcpyAsync(c.data(), csum_.p, sizeof(R) * c.size(), cudaMemcpyDeviceToHost, stream));
    MPM_CUDA(cudaMemcpyAsync(tg.data(), target_.p, sizeof(R) * tg.size(), cudaMemcpyDeviceToHost, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
    double L = 0;
    for (int t = 0; t <= steps_; ++t) {
      if (loss_w_[t] == 0.0) continue;
      for (size_t q = 0; q < (size_t)E_ * D; ++q) {
        const double e = (double)(c[(size_t)t * E_ * D + q] / (R)pw_sum_) - (double)tg[(size_t)t * E_ * D + q];
        L += loss_w_[t] * e * e;
      }
    }
    return L;
  }

  // ---------------------------------------------------------------- reverse
  void backward() override {
    MPM_REQUIRE(fwd_done_, "cls_mpm_backward before a forward rollout");
    const int steps = steps_;
    const int n_seg = (steps + K_ - 1) / K_;
    const Phys<R> c = phys();
    auto seed = [&](AdjArgs<R>& a, int t) {
      a.seed_w = (R)loss_w_[t];
      a.csum = csum_.p + (size_t)t * E_ * D;
      a.target = target_.p + (size_t)t * E_ * D;
      a.pw_sum = (R)pw_sum_;
    };
    auto g2pT = [&](AdjArgs<R>& a, int h) {
      const int sh = h / K_, kh = h - sh * K_;
      a.x_h = rx(sh, kh);
      a.gv_h = gv(sh % 2, kh);
      a.gacc = gacc_.p;
    };
    timed(MK_OTHER, [&] { cudaMemsetAsync(gact_.p, 0, sizeof(R) * gact_.n, stream); });
    recompute(n_seg - 1);
    int cur = 0;
    {  // G2P^T of the last step, seeded by the loss at step `steps`
      AdjArgs<R> a;
      std::memset(&a, 0, sizeof(a));
      a.c = c;
      seed(a, steps);
      g2pT(a, steps - 1);
      a.ax_out = AX_[0].p; a.aF_out = AF_[0].p;
      launch_adj(2, a);
    }
    for (int f = steps - 1; f >= 0; --f) {
      const int s = f / K_, k = f - s * K_;
      if (f >= 1 && k == 0) recompute(s - 1);
      timed(MK_GADJ, [&] {
        mpm_grid_adj_kernel<R, D><<<grid_dims(), 256, 0, stream>>>(c, gacc_.p, gv(s % 2, k), ga_.p,
                                                                   bbox(s % 2, k));
      });
      AdjArgs<R> a;
      std::memset(&a, 0, sizeof(a));
      a.c = c;
      a.x_f = rx(s, k); a.v_f = rv(s, k); a.C_f = rC(s, k); a.F_f = rF(s, k);
      a.act_f = act(f);
      a.ga = ga_.p;
      a.ax_in = AX_[cur].p; a.aF_in = AF_[cur].p;
      a.gact = gact_.p + (size_t)f * E_ * M_;
      seed(a, f);
      if (f >= 1) {
        g2pT(a, f - 1);
        a.ax_out = AX_[1 - cur].p; a.aF_out = AF_[1 - cur].p;
        launch_adj(3, a);
        cur = 1 - cur;
      } else {
        a.out_ax = out_ax_.p; a.out_av = out_av_.p; a.out_aC = out_aC_.p; a.out_aF = out_aF_.p;
        launch_adj(1, a);
      }
    }
    MPM_CUDA(cudaGetLastError());
    bwd_done_ = true;
  }

  void graph_capture(int steps) override {
    MPM_REQUIRE(stream != nullptr, "graph capture needs a non-default stream");
    MPM_REQUIRE(!prof_.on, "disable profiling before graph capture");
    if (gexec_) { cudaGraphExecDestroy(gexec_); gexec_ = nullptr; }
    if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
    MPM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      forward(steps);
      backward();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    MPM_CUDA(cudaStreamEndCapture(stream, &graph_));
    MPM_CUDA(cudaGraphInstantiate(&gexec_, graph_, 0));
  }

  void graph_launch() override {
    MPM_REQUIRE(gexec_ != nullptr, "no captured graph");
    MPM_CUDA(cudaGraphLaunch(gexec_, stream));
  }

  // ------------------------------------------------------------------- I/O
  // user layout [E][P][comps] (double) <-> planes [comps][E][P_internal] (R)
  void up_planes(const double* h, R* d, int comps) {
    const size_t EP = (size_t)E_ * P_;
    std::vector<R> tmp(EP * comps);
    for (int e = 0; e < E_; ++e)
      for (int i = 0; i < P_; ++i) {
        const double* src = h + ((size_t)e * P_ + perm_[i]) * comps;
        for (int k = 0; k < comps; ++k) tmp[(size_t)k * EP + (size_t)e * P_ + i] = (R)src[k];
      }
    MPM_CUDA(cudaMemcpyAsync(d, tmp.data(), sizeof(R) * tmp.size(), cudaMemcpyHostToDevice, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
  }
  void down_planes(const R* d, double* h, int comps) {
    const size_t EP = (size_t)E_ * P_;
    std::vector<R> tmp(EP * comps);
    MPM_CUDA(cudaMemcpyAsync(tmp.data(), d, sizeof(R) * tmp.size(), cudaMemcpyDeviceToHost, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
    for (int e = 0; e < E_; ++e)
      for (int i = 0; i < P_; ++i) {
        double* dst = h + ((size_t)e * P_ + perm_[i]) * comps;
        for (int k = 0; k < comps; ++k) dst[k] = (double)tmp[(size_t)k * EP + (size_t)e * P_ + i];
      }
  }
  void up(const double* h, R* d, size_t n) {
    std::vector<R> tmp(n);
    for (size_t i = 0; i < n; ++i) tmp[i] = (R)h[i];
    MPM_CUDA(cudaMemcpyAsync(d, tmp.data(), sizeof(R) * n, cudaMemcpyHostToDevice, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
  }
  void down(const R* d, double* h, size_t n) {
    std::vector<R> tmp(n);
    MPM_CUDA(cudaMemcpyAsync(tmp.data(), d, sizeof(R) * n, cudaMemcpyDeviceToHost, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
    for (size_t i = 0; i < n; ++i) h[i] = (double)tmp[i];
  }

  void set_state(const double* x0, const double* v0) override {
    MPM_REQUIRE(x0 != nullptr, "x0 required");
    up_planes(x0, ckx(0), D);
    if (v0) up_planes(v0, ckv(0), D);
    else MPM_CUDA(cudaMemsetAsync(ckv(0), 0, sizeof(R) * VX(), stream));
    MPM_CUDA(cudaMemsetAsync(ckC(0), 0, sizeof(R) * VM(), stream));
    std::vector<R> eye(VM(), R(0));
    for (int d = 0; d < D; ++d)
      for (size_t q = 0; q < (size_t)E_ * P_; ++q) eye[(size_t)(d * D + d) * E_ * P_ + q] = R(1);
    MPM_CUDA(cudaMemcpyAsync(ckF(0), eye.data(), sizeof(R) * eye.size(), cudaMemcpyHostToDevice, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
    fwd_done_ = bwd_done_ = false;
  }

  void set_actuation(const double* act_h) override { up(act_h, act_.p, (size_t)T_ * E_ * M_); }

  void set_loss(const double* w, const double* target, const double* pw) override {
    if (w) loss_w_.assign(w, w + T_ + 1);
    if (target) up(target, target_.p, (size_t)(T_ + 1) * E_ * D);
    if (pw) {
      std::vector<double> pi(P_);
      pw_sum_ = 0;
      for (int i = 0; i < P_; ++i) {
        pi[i] = pw[perm_[i]];
        pw_sum_ += pw[i];
      }
      MPM_REQUIRE(pw_sum_ > 0, "particle weights must have a positive sum");
      up(pi.data(), pw_.p, P_);
    }
  }

  void final_state(double* x, double* v, double* C, double* F) override {
    MPM_REQUIRE(fwd_done_, "no rollout yet");
    if (x) down_planes(fin_x_.p, x, D);
    if (v) down_planes(fin_v_.p, v, D);
    if (C) down_planes(fin_C_.p, C, D * D);
    if (F) down_planes(fin_F_.p, F, D * D);
  }

  void grads(double* gact, double* gx0, double* gv0, double* gC0, double* gF0) override {
    MPM_REQUIRE(bwd_done_, "no reverse pass yet");
    if (gact) down(gact_.p, gact, (size_t)T_ * E_ * M_);
    if (gx0) down_planes(out_ax_.p, gx0, D);
    if (gv0) down_planes(out_av_.p, gv0, D);
    if (gC0) down_planes(out_aC_.p, gC0, D * D);
    if (gF0) down_planes(out_aF_.p, gF0, D * D);
  }

  void centers(double* c) override {
    down(csum_.p, c, (size_t)(T_ + 1) * E_ * D);
    for (size_t i = 0; i < (size_t)(T_ + 1) * E_ * D; ++i) c[i] /= pw_sum_;
  }

  void profile_enable(bool on) override {
    MPM_CUDA(prof_.collect(stream));
    prof_.on = on;
  }
  void profile_read(double* ms, long long* launches, bool reset) override {
    MPM_CUDA(prof_.collect(stream));
    prof_.read(ms, launches, reset);
  }

 private:
  cls_mpm_params p_;
  int E_ = 0, P_ = 0, M_ = 1, T_ = 0, K_ = 1, n_grid_ = 0, nb_ = 0, n_chunks_ = 0, slots_ = 2;
  int tile_cap_ = 0, sm_mode_ = 0, steps_ = 0;
  long long nblk_ = 0;
  size_t n_ckpt_ = 0, fwd_smem_ = 0, adj_smem_ = 0;
  double pw_sum_ = 1;
  std::vector<double> loss_w_;
  std::vector<int> perm_;  // internal particle -> user particle
  std::vector<int> chunk_start_h_, chunk_len_h_;
  bool runs_ = false;  // CLS_MPM_ORDER_BASE_RUNS
  bool fwd_done_ = false, bwd_done_ = false;
  Buf<R> ck_x_, ck_v_, ck_C_, ck_F_;
  Buf<R> X_[2], Fw_[2], RX_[2], RV_[2], RC_[2], RF_[2], AX_[2], AF_[2];
  Buf<V> gv_[2], acc_, gacc_, ga_;
  Buf<int> bboxes_, muscle_, chunk_start_, chunk_len_;
  Buf<R> fin_x_, fin_v_, fin_C_, fin_F_, out_ax_, out_av_, out_aC_, out_aF_;
  Buf<R> act_, gact_, csum_, target_, fibre_, pw_;
  EventProfile<MK_COUNT> prof_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t gexec_ = nullptr;
};

}  // namespace mpm
}  // namespace cls

struct cls_mpm {
  std::unique_ptr<cls::mpm::MpmBase> impl;
};

template <typename F>
static int mguard(cls_mpm* s, F&& f) {
  if (!s || !s->impl) return CLS_ERR_INVALID;
  try {
    f(*s->impl);
    return CLS_OK;
  } catch (const cls::mpm::MFail& e) {
    s->impl->err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    s->impl->err = e.what();
    return CLS_ERR_INVALID;
  }
}

extern "C" {

void cls_mpm_default_params(cls_mpm_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_steps = 1000;
  p->n_grid = 32;
  p->bound = 3;
  p->material = CLS_MPM_FIXED_COROTATED;
  p->precision = 32;
  p->checkpoint_every = 50;
  p->dt = 1e-3;
  p->gravity = -10.0;
  p->p_vol = 1.0;
  p->mu = 40.0;
  p->la = 40.0;
  p->act_strength = 4.0;
  p->mass = 1.0;
  p->particle_order = CLS_MPM_ORDER_BASE_RUNS;
}

int cls_mpm_create(const cls_mpm_body* body, const cls_mpm_params* params, int32_t n_envs,
                   cls_mpm** out) {
  using namespace cls::mpm;
  if (!out) return CLS_ERR_INVALID;
  *out = nullptr;
  try {
    MPM_REQUIRE(body && params && n_envs > 0, "null argument or no envs");
    MPM_REQUIRE(body->dim == 2 || body->dim == 3, "dim must be 2 or 3");
    MPM_REQUIRE(body->n_particles > 0 && body->positions, "no particles");
    MPM_REQUIRE(params->n_grid >= 8 && params->max_steps >= 1, "bad grid or horizon");
    MPM_REQUIRE(params->material == CLS_MPM_NEO_HOOKEAN || body->dim == 2,
                "fixed-corotated is available in 2D only");
    MPM_REQUIRE(params->precision == 32 || params->precision == 64, "precision must be 32 or 64");
    for (int q = 0; q < body->n_particles * body->dim; ++q) {
      const double c = body->positions[q];
      MPM_REQUIRE(c * params->n_grid >= 1.0 && c * params->n_grid <= params->n_grid - 2.0,
                  "particles must start inside the grid (one cell from every side)");
    }
    auto* s = new cls_mpm;
    try {
      if (params->precision == 32) {
        if (body->dim == 2) s->impl.reset(new MpmImpl<float, 2>(*body, *params, n_envs));
        else s->impl.reset(new MpmImpl<float, 3>(*body, *params, n_envs));
      } else {
        if (body->dim == 2) s->impl.reset(new MpmImpl<double, 2>(*body, *params, n_envs));
        else s->impl.reset(new MpmImpl<double, 3>(*body, *params, n_envs));
      }
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
    return CLS_OK;
  } catch (const MFail& e) {
    g_mpm_create_error = e.msg;
    return e.code;
  }
}

int cls_mpm_destroy(cls_mpm* s) {
  if (!s) return CLS_ERR_INVALID;
  delete s;
  return CLS_OK;
}

const char* cls_mpm_last_error(const cls_mpm* s) {
  if (!s || !s->impl) return cls::mpm::g_mpm_create_error.c_str();
  return s->impl->err.c_str();
}

int cls_mpm_set_stream(cls_mpm* s, void* stream) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.stream = (cudaStream_t)stream; });
}
int cls_mpm_set_state(cls_mpm* s, const double* x0, const double* v0) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.set_state(x0, v0); });
}
int cls_mpm_set_actuation(cls_mpm* s, const double* act) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.set_actuation(act); });
}
int cls_mpm_set_loss(cls_mpm* s, const double* w, const double* target, const double* pw) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.set_loss(w, target, pw); });
}
int cls_mpm_forward(cls_mpm* s, int32_t steps) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.forward(steps); });
}
int cls_mpm_loss(cls_mpm* s, double* loss) {
  return mguard(s, [&](cls::mpm::MpmBase& b) {
    const double L = b.loss();
    if (loss) *loss = L;
  });
}
int cls_mpm_backward(cls_mpm* s) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.backward(); });
}
int cls_mpm_get_final_state(cls_mpm* s, double* x, double* v, double* C, double* F) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.final_state(x, v, C, F); });
}
int cls_mpm_get_grads(cls_mpm* s, double* gact, double* gx0, double* gv0, double* gC0, double* gF0) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.grads(gact, gx0, gv0, gC0, gF0); });
}
int cls_mpm_get_centers(cls_mpm* s, double* centers) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.centers(centers); });
}
int cls_mpm_graph_capture(cls_mpm* s, int32_t steps) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.graph_capture(steps); });
}
int cls_mpm_graph_launch(cls_mpm* s) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.graph_launch(); });
}
int cls_mpm_profile_enable(cls_mpm* s, int32_t on) {
  return mguard(s, [&](cls::mpm::MpmBase& b) { b.profile_enable(on != 0); });
}
// Calibration of the scatter roofline: 16-byte vector reductions
// (red.global.add.v4.f32, the P2G / G2P^T scatter instruction) from every
// thread into a buffer of n_nodes 16-byte nodes, each warp's 32 lanes on 32
// distinct nodes of a pseudo-random 1 KB block walk -- the pattern of the
// particle kernels' scatters, where a warp's lanes hold particles of distinct
// cells and successive stencil offsets move to neighbouring nodes.
namespace {
__global__ void mpm_red_peak_kernel(cls::V4<float>* __restrict__ nodes, long long n_nodes, int per_thread) {
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  const unsigned long long warp = tid >> 5, lane = tid & 31;
  const long long nblk = n_nodes / 64;
  unsigned long long h = warp * 0x9E3779B97F4A7C15ULL + 1;
  for (int k = 0; k < per_thread; ++k) {
    if ((k & 7) == 0) h = h * 6364136223846793005ULL + 1442695040888963407ULL;
    const long long blk = (long long)((h >> 20) % (unsigned long long)nblk);
    const long long node = blk * 64 + (long long)((lane * 2 + (k & 7)) & 63);
    cls::mpm::red4<float>(nodes + node, 1.f, 1.f, 1.f, 1.f);
  }
}
}  // namespace

int cls_mpm_reduction_peak(int64_t n_nodes, int64_t n_ops, double* ops_per_s) {
  if (!ops_per_s || n_nodes < 64 || n_ops < 1) return CLS_ERR_INVALID;
  cls::V4<float>* buf = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = CLS_OK;
  const int per_thread = 64, threads = 256;
  const long long n_threads = (n_ops + per_thread - 1) / per_thread;
  const int blocks = (int)std::min<long long>((n_threads + threads - 1) / threads, 1LL << 30);
  if (cudaMalloc(&buf, sizeof(cls::V4<float>) * (size_t)n_nodes) != cudaSuccess) return CLS_ERR_OOM;
  float ms = 0.f;
  if (cudaMemset(buf, 0, sizeof(cls::V4<float>) * (size_t)n_nodes) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = CLS_ERR_CUDA;
  } else {
    mpm_red_peak_kernel<<<blocks, threads>>>(buf, n_nodes, per_thread);  // warm-up
    cudaEventRecord(e0);
    mpm_red_peak_kernel<<<blocks, threads>>>(buf, n_nodes, per_thread);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
        cudaGetLastError() != cudaSuccess)
      rc = CLS_ERR_CUDA;
  }
  if (rc == CLS_OK) *ops_per_s = (double)blocks * threads * per_thread / (ms * 1e-3);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  return rc;
}

int cls_mpm_profile_read(cls_mpm* s, double* ms, int64_t* launches, int32_t reset) {
  return mguard(s, [&](cls::mpm::MpmBase& b) {
    b.profile_read(ms, reinterpret_cast<long long*>(launches), reset != 0);
  });
}

}  // extern "C"
