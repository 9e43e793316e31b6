// mpm_runtime.cu -- cls_mpm_* C ABI: MLS-MPM episodes with checkpointed
// reverse passes (forward keeps a checkpoint every K steps; the reverse pass
// recomputes each segment, then for every step rebuilds its grid and runs the
// adjoint kernels, as the reference's advance_core_grad does per step).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cls_b200.h"
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
};

template <typename R, int D>
class MpmImpl final : public MpmBase {
 public:
  MpmImpl(const cls_mpm_body& b, const cls_mpm_params& p, int n_envs) : p_(p) {
    E_ = n_envs;
    P_ = b.n_particles;
    M_ = std::max(1, b.n_muscles);
    T_ = p.max_steps;
    K_ = std::max(1, p.checkpoint_every);
    n_grid_ = p.n_grid;
    cells_ = 1;
    for (int d = 0; d < D; ++d) cells_ *= n_grid_;
    const size_t EP = (size_t)E_ * P_;
    n_ckpt_ = (T_ + K_ - 1) / K_ + 1;
    ck_x_.alloc(n_ckpt_ * EP * D); ck_v_.alloc(n_ckpt_ * EP * D);
    ck_C_.alloc(n_ckpt_ * EP * D * D); ck_F_.alloc(n_ckpt_ * EP * D * D);
    rc_x_.alloc((K_ + 1) * EP * D); rc_v_.alloc((K_ + 1) * EP * D);
    rc_C_.alloc((K_ + 1) * EP * D * D); rc_F_.alloc((K_ + 1) * EP * D * D);
    for (int s = 0; s < 2; ++s) {
      ax_[s].alloc(EP * D); av_[s].alloc(EP * D); aC_[s].alloc(EP * D * D); aF_[s].alloc(EP * D * D);
    }
    fin_x_.alloc(EP * D); fin_v_.alloc(EP * D); fin_C_.alloc(EP * D * D); fin_F_.alloc(EP * D * D);
    gm_.alloc((size_t)E_ * cells_); gmv_.alloc((size_t)E_ * cells_ * D); gvo_.alloc((size_t)E_ * cells_ * D);
    g_gvo_.alloc((size_t)E_ * cells_ * D); g_gv_.alloc((size_t)E_ * cells_ * D); g_gm_.alloc((size_t)E_ * cells_);
    act_.alloc((size_t)T_ * E_ * M_); gact_.alloc((size_t)T_ * E_ * M_);
    center_.alloc((size_t)(T_ + 1) * E_ * D);
    target_.alloc((size_t)(T_ + 1) * E_ * D);
    muscle_.alloc(P_); fibre_.alloc((size_t)P_ * D); pw_.alloc(P_);
    stage_.alloc(std::max<size_t>({(size_t)T_ * E_ * M_, EP * D * D, (size_t)(T_ + 1) * E_ * D, (size_t)P_ * D}));
    std::vector<int> mus(b.muscle ? b.muscle : nullptr, b.muscle ? b.muscle + P_ : nullptr);
    if (mus.empty()) mus.assign(P_, -1);
    for (int m : mus) MPM_REQUIRE(m >= -1 && m < M_, "muscle index out of range");
    MPM_CUDA(cudaMemcpy(muscle_.p, mus.data(), sizeof(int) * P_, cudaMemcpyHostToDevice));
    std::vector<R> fib((size_t)P_ * D, R(0));
    for (int q = 0; q < P_; ++q)
      for (int d = 0; d < D; ++d)
        fib[(size_t)q * D + d] = b.fibre ? (R)b.fibre[(size_t)q * D + d] : (d == 1 ? R(1) : R(0));
    MPM_CUDA(cudaMemcpy(fibre_.p, fib.data(), sizeof(R) * fib.size(), cudaMemcpyHostToDevice));
    std::vector<R> pw(P_, R(1));
    pw_sum_ = P_;
    MPM_CUDA(cudaMemcpy(pw_.p, pw.data(), sizeof(R) * P_, cudaMemcpyHostToDevice));
    loss_w_.assign(T_ + 1, 0.0);
    MPM_CUDA(cudaMemset(act_.p, 0, sizeof(R) * act_.n));
    MPM_CUDA(cudaMemset(target_.p, 0, sizeof(R) * target_.n));
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

  Args<R> base_args() const {
    Args<R> a;
    std::memset(&a, 0, sizeof(a));
    a.n_envs = E_; a.P = P_; a.M = M_; a.n_grid = n_grid_; a.bound = p_.bound; a.material = p_.material;
    a.cells = cells_;
    a.dx = (R)(1.0 / n_grid_); a.inv_dx = (R)n_grid_; a.dt = (R)p_.dt;
    a.ks = (R)(p_.dt * p_.p_vol * 4.0 * n_grid_ * n_grid_);
    a.mu = (R)p_.mu; a.la = (R)p_.la; a.act_strength = (R)p_.act_strength;
    a.gravity = (R)p_.gravity; a.mass = (R)p_.mass;
    a.muscle = muscle_.p; a.fibre = fibre_.p;
    a.gm = gm_.p; a.gmv = gmv_.p; a.gvo = gvo_.p;
    a.g_gvo = g_gvo_.p; a.g_gv = g_gv_.p; a.g_gm = g_gm_.p;
    return a;
  }

  size_t EP() const { return (size_t)E_ * P_; }
  static int blocks(long long n) { return (int)std::max<long long>(1, std::min<long long>(148 * 32, (n + 255) / 256)); }

  // one forward step from (x, v, C, F) to (x1, v1, C1, F1)
  void step(const R* x, const R* v, const R* C, const R* F, R* x1, R* v1, R* C1, R* F1, int f, bool write_F) {
    Args<R> a = base_args();
    a.x = x; a.v = v; a.C = C; a.F = F; a.x1 = x1; a.v1 = v1; a.C1 = C1; a.F1 = F1;
    a.act = act_.p + (size_t)f * E_ * M_;
    MPM_CUDA(cudaMemsetAsync(gm_.p, 0, sizeof(R) * gm_.n, stream));
    MPM_CUDA(cudaMemsetAsync(gmv_.p, 0, sizeof(R) * gmv_.n, stream));
    p2g_kernel<R, D><<<blocks(EP()), 256, 0, stream>>>(a, write_F ? 1 : 0);
    grid_op_kernel<R, D><<<blocks((long long)E_ * cells_), 256, 0, stream>>>(a);
    if (x1) g2p_kernel<R, D><<<blocks(EP()), 256, 0, stream>>>(a);
    launches_ += x1 ? 3 : 2;
  }

  void center_at(const R* x, int t) {
    center_kernel<R, D><<<E_, 256, 0, stream>>>(x, pw_.p, (R)pw_sum_, P_, center_.p + (size_t)t * E_ * D);
    launches_ += 1;
  }

  R* slot(Buf<R>& b, size_t per, int i) { return b.p + per * i; }

  void forward(int steps) override {
    MPM_REQUIRE(steps >= 1 && steps <= T_, "steps must be in [1, max_steps]");
    steps_ = steps;
    const size_t px = EP() * D, pm = EP() * D * D;
    // working states live in the record buffers' slots 0 and 1 (ping-pong);
    // checkpoint slot 0 holds the initial state
    MPM_CUDA(cudaMemcpyAsync(slot(rc_x_, px, 0), ck_x_.p, sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaMemcpyAsync(slot(rc_v_, px, 0), ck_v_.p, sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaMemcpyAsync(slot(rc_C_, pm, 0), ck_C_.p, sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaMemcpyAsync(slot(rc_F_, pm, 0), ck_F_.p, sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
    int cur = 0;
    for (int f = 0; f < steps; ++f) {
      const int nx = 1 - cur;
      if (f > 0 && f % K_ == 0) {
        const int s = f / K_;
        MPM_CUDA(cudaMemcpyAsync(slot(ck_x_, px, s), slot(rc_x_, px, cur), sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
        MPM_CUDA(cudaMemcpyAsync(slot(ck_v_, px, s), slot(rc_v_, px, cur), sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
        MPM_CUDA(cudaMemcpyAsync(slot(ck_C_, pm, s), slot(rc_C_, pm, cur), sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
        MPM_CUDA(cudaMemcpyAsync(slot(ck_F_, pm, s), slot(rc_F_, pm, cur), sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
      }
      center_at(slot(rc_x_, px, cur), f);
      step(slot(rc_x_, px, cur), slot(rc_v_, px, cur), slot(rc_C_, pm, cur), slot(rc_F_, pm, cur),
           slot(rc_x_, px, nx), slot(rc_v_, px, nx), slot(rc_C_, pm, nx), slot(rc_F_, pm, nx), f, true);
      cur = nx;
    }
    center_at(slot(rc_x_, px, cur), steps);
    final_slot_ = cur;
    // keep the final state outside the record buffers
    MPM_CUDA(cudaMemcpyAsync(fin_x_.p, slot(rc_x_, px, cur), sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaMemcpyAsync(fin_v_.p, slot(rc_v_, px, cur), sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaMemcpyAsync(fin_C_.p, slot(rc_C_, pm, cur), sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaMemcpyAsync(fin_F_.p, slot(rc_F_, pm, cur), sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
    MPM_CUDA(cudaGetLastError());
    fwd_done_ = true;
  }

  double loss() override {
    MPM_REQUIRE(fwd_done_, "cls_mpm_loss before a forward rollout");
    std::vector<R> c((size_t)(steps_ + 1) * E_ * D), tg((size_t)(steps_ + 1) * E_ * D);
    MPM_CUDA(cudaMemcpyAsync(c.data(), center_.p, sizeof(R) * c.size(), cudaMemcpyDeviceToHost, stream));
    MPM_CUDA(cudaMemcpyAsync(tg.data(), target_.p, sizeof(R) * tg.size(), cudaMemcpyDeviceToHost, stream));
    MPM_CUDA(cudaStreamSynchronize(stream));
    double L = 0;
    for (int t = 0; t <= steps_; ++t) {
      if (loss_w_[t] == 0.0) continue;
      for (size_t q = 0; q < (size_t)E_ * D; ++q) {
        const double e = (double)c[(size_t)t * E_ * D + q] - (double)tg[(size_t)t * E_ * D + q];
        L += loss_w_[t] * e * e;
      }
    }
    return L;
  }

  void seed(R* ax, int t) {
    if (loss_w_[t] == 0.0) return;
    seed_kernel<R, D><<<blocks(EP()), 256, 0, stream>>>(ax, center_.p + (size_t)t * E_ * D,
                                                       target_.p + (size_t)t * E_ * D, pw_.p,
                                                       (R)loss_w_[t], (R)pw_sum_, E_, P_);
    launches_ += 1;
  }

  void backward() override {
    MPM_REQUIRE(fwd_done_, "cls_mpm_backward before a forward rollout");
    const size_t px = EP() * D, pm = EP() * D * D;
    int a = 0;  // adjoint buffers: a = state t + 1, 1 - a = state t
    MPM_CUDA(cudaMemsetAsync(ax_[a].p, 0, sizeof(R) * px, stream));
    MPM_CUDA(cudaMemsetAsync(av_[a].p, 0, sizeof(R) * px, stream));
    MPM_CUDA(cudaMemsetAsync(aC_[a].p, 0, sizeof(R) * pm, stream));
    MPM_CUDA(cudaMemsetAsync(aF_[a].p, 0, sizeof(R) * pm, stream));
    MPM_CUDA(cudaMemsetAsync(gact_.p, 0, sizeof(R) * gact_.n, stream));
    seed(ax_[a].p, steps_);
    const int n_seg = (steps_ + K_ - 1) / K_;
    for (int s = n_seg - 1; s >= 0; --s) {
      const int t0 = s * K_, t1 = std::min(t0 + K_, steps_);
      // recompute the segment's states into record slots 0 .. t1 - t0 - 1
      MPM_CUDA(cudaMemcpyAsync(slot(rc_x_, px, 0), slot(ck_x_, px, s), sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
      MPM_CUDA(cudaMemcpyAsync(slot(rc_v_, px, 0), slot(ck_v_, px, s), sizeof(R) * px, cudaMemcpyDeviceToDevice, stream));
      MPM_CUDA(cudaMemcpyAsync(slot(rc_C_, pm, 0), slot(ck_C_, pm, s), sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
      MPM_CUDA(cudaMemcpyAsync(slot(rc_F_, pm, 0), slot(ck_F_, pm, s), sizeof(R) * pm, cudaMemcpyDeviceToDevice, stream));
      for (int f = t0; f < t1 - 1; ++f) {
        const int k = f - t0;
        step(slot(rc_x_, px, k), slot(rc_v_, px, k), slot(rc_C_, pm, k), slot(rc_F_, pm, k),
             slot(rc_x_, px, k + 1), slot(rc_v_, px, k + 1), slot(rc_C_, pm, k + 1), slot(rc_F_, pm, k + 1),
             f, true);
      }
      for (int f = t1 - 1; f >= t0; --f) {
        const int k = f - t0;
        const R* x = slot(rc_x_, px, k);
        const R* v = slot(rc_v_, px, k);
        const R* C = slot(rc_C_, pm, k);
        const R* F = slot(rc_F_, pm, k);
        step(x, v, C, F, nullptr, nullptr, nullptr, nullptr, f, false);  // grid of step f
        Args<R> ar = base_args();
        ar.x = x; ar.v = v; ar.C = C; ar.F = F;
        ar.act = act_.p + (size_t)f * E_ * M_;
        ar.gact = gact_.p + (size_t)f * E_ * M_;
        ar.ax = ax_[a].p; ar.av = av_[a].p; ar.aC = aC_[a].p; ar.aF = aF_[a].p;
        ar.nx = ax_[1 - a].p; ar.nv = av_[1 - a].p; ar.nC = aC_[1 - a].p; ar.nF = aF_[1 - a].p;
        MPM_CUDA(cudaMemsetAsync(g_gvo_.p, 0, sizeof(R) * g_gvo_.n, stream));
        g2p_adj_kernel<R, D><<<blocks(EP()), 256, 0, stream>>>(ar);
        grid_op_adj_kernel<R, D><<<blocks((long long)E_ * cells_), 256, 0, stream>>>(ar);
        p2g_adj_kernel<R, D><<<blocks(EP()), 256, 0, stream>>>(ar);
        launches_ += 3;
        a = 1 - a;
        seed(ax_[a].p, f);
      }
    }
    adj_slot_ = a;
    MPM_CUDA(cudaGetLastError());
    bwd_done_ = true;
  }

  void graph_capture(int steps) override {
    MPM_REQUIRE(stream != nullptr, "graph capture needs a non-default stream");
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
  void up(const double* h, R* d, size_t n) {
    MPM_REQUIRE(n <= stage_.n, "staging too small");
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
    const size_t px = EP() * D, pm = EP() * D * D;
    MPM_REQUIRE(x0 != nullptr, "x0 required");
    up(x0, ck_x_.p, px);
    if (v0) up(v0, ck_v_.p, px);
    else MPM_CUDA(cudaMemsetAsync(ck_v_.p, 0, sizeof(R) * px, stream));
    MPM_CUDA(cudaMemsetAsync(ck_C_.p, 0, sizeof(R) * pm, stream));
    std::vector<double> eye(pm, 0.0);
    for (size_t q = 0; q < EP(); ++q)
      for (int d = 0; d < D; ++d) eye[q * D * D + d * D + d] = 1.0;
    up(eye.data(), ck_F_.p, pm);
    fwd_done_ = bwd_done_ = false;
  }

  void set_actuation(const double* act) override { up(act, act_.p, (size_t)T_ * E_ * M_); }

  void set_loss(const double* w, const double* target, const double* pw) override {
    if (w) loss_w_.assign(w, w + T_ + 1);
    if (target) up(target, target_.p, (size_t)(T_ + 1) * E_ * D);
    if (pw) {
      up(pw, pw_.p, P_);
      pw_sum_ = 0;
      for (int q = 0; q < P_; ++q) pw_sum_ += pw[q];
      MPM_REQUIRE(pw_sum_ > 0, "particle weights must have a positive sum");
    }
  }

  void final_state(double* x, double* v, double* C, double* F) override {
    MPM_REQUIRE(fwd_done_, "no rollout yet");
    const size_t px = EP() * D, pm = EP() * D * D;
    if (x) down(fin_x_.p, x, px);
    if (v) down(fin_v_.p, v, px);
    if (C) down(fin_C_.p, C, pm);
    if (F) down(fin_F_.p, F, pm);
  }

  void grads(double* gact, double* gx0, double* gv0, double* gC0, double* gF0) override {
    MPM_REQUIRE(bwd_done_, "no reverse pass yet");
    const size_t px = EP() * D, pm = EP() * D * D;
    if (gact) down(gact_.p, gact, (size_t)T_ * E_ * M_);
    if (gx0) down(ax_[adj_slot_].p, gx0, px);
    if (gv0) down(av_[adj_slot_].p, gv0, px);
    if (gC0) down(aC_[adj_slot_].p, gC0, pm);
    if (gF0) down(aF_[adj_slot_].p, gF0, pm);
  }

  void centers(double* c) override { down(center_.p, c, (size_t)(T_ + 1) * E_ * D); }

  long long launches_ = 0;

 private:
  cls_mpm_params p_;
  int E_ = 0, P_ = 0, M_ = 1, T_ = 0, K_ = 1, n_grid_ = 0, steps_ = 0, final_slot_ = 0, adj_slot_ = 0;
  long long cells_ = 0;
  size_t n_ckpt_ = 0;
  double pw_sum_ = 1;
  std::vector<double> loss_w_;
  bool fwd_done_ = false, bwd_done_ = false;
  Buf<R> ck_x_, ck_v_, ck_C_, ck_F_, rc_x_, rc_v_, rc_C_, rc_F_;
  Buf<R> ax_[2], av_[2], aC_[2], aF_[2];
  Buf<R> gm_, gmv_, gvo_, g_gvo_, g_gv_, g_gm_, act_, gact_, center_, target_, fibre_, pw_, stage_;
  Buf<int> muscle_;
  Buf<R> fin_x_, fin_v_, fin_C_, fin_F_;
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

}  // extern "C"
