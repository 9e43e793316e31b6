// ms_runtime.cu -- the cls_* C ABI: batch packing, device buffers, the
// checkpointed forward / reverse schedule and CUDA-graph capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/cls_b200.h"
#include "cls_profile.cuh"
#include "ms_dense_host.h"
#include "ms_env_host.h"
#include "ms_sched.h"
#include "ms_segment.cuh"

// threads of the batched controller's step kernels (one CTA per env)
#ifndef CLS_STEP_THREADS
#define CLS_STEP_THREADS 128
#endif

namespace cls {

static thread_local std::string g_create_error;

struct Fail {
  int code;
  std::string msg;
};

#define CLS_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw Fail{e_ == cudaErrorMemoryAllocation ? CLS_ERR_OOM : CLS_ERR_CUDA,          \
                 std::string(#call) + ": " + cudaGetErrorString(e_)};                   \
  } while (0)

#define CLS_REQUIRE(cond, msg)                                                          \
  do {                                                                                  \
    if (!(cond)) throw Fail{CLS_ERR_INVALID, (msg)};                                    \
  } while (0)

static inline int round4(int x) { return (x + 3) & ~3; }

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free();
    n = count;
    if (count) CLS_CUDA(cudaMalloc(&p, sizeof(T) * count));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { free(); }
};

// ------------------------------------------------------------ host-side pack
struct HostRobot {
  int n_v = 0, n_s = 0, n_out = 0, n_c = 0, pos_pad = 0, robot_id = -1, n_layers = 0;
  int width[kMaxLayers + 1] = {0};
  int full_cols[kMaxLayers] = {0};
  std::vector<double> objects;           // [n_v][3]
  std::vector<int> sa, sb, out;          // per spring
  std::vector<double> len, stiff, coef;  // per spring (stiffness scaled)
};

// launch categories for the per-kernel CUDA-event profile
enum ProfKind : int {
  PK_FWD = 0, PK_RECOMP, PK_REV, PK_WGRAD, PK_LOSS, PK_ADAM, PK_OTHER,
  PK_CGEMM,      // batched controller: forward GEMMs (first pass and recompute)
  PK_CGEMM_ADJ,  // batched controller: adjoint GEMMs
  PK_COUNT
};

using Profiler = EventProfile<PK_COUNT>;

// Pinned host -> device staging ring for small per-launch tables: slot k's
// host bytes are reused only after the event recorded behind its last copy
// has completed, so uploads never block on the stream.
struct StageRing {
  static constexpr int kSlots = 32;
  size_t bytes = 0;
  unsigned char* host = nullptr;
  unsigned char* dev = nullptr;
  cudaEvent_t ev[kSlots] = {};
  bool used[kSlots] = {};
  int next = 0;
  cudaError_t init(size_t b) {
    bytes = (b + 255) & ~size_t(255);
    cudaError_t r = cudaMallocHost(&host, bytes * kSlots);
    if (r != cudaSuccess) return r;
    r = cudaMalloc(&dev, bytes * kSlots);
    if (r != cudaSuccess) return r;
    for (int k = 0; k < kSlots; ++k) {
      r = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
      if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
  }
  ~StageRing() {
    for (int k = 0; k < kSlots; ++k)
      if (ev[k]) cudaEventDestroy(ev[k]);
    if (host) cudaFreeHost(host);
    if (dev) cudaFree(dev);
  }
  // host and device addresses of the next free slot
  cudaError_t acquire(unsigned char** h, unsigned char** d, int* slot) {
    const int k = next;
    next = (next + 1) % kSlots;
    if (used[k]) {
      const cudaError_t r = cudaEventSynchronize(ev[k]);
      if (r != cudaSuccess) return r;
    }
    *h = host + (size_t)k * bytes;
    *d = dev + (size_t)k * bytes;
    *slot = k;
    return cudaSuccess;
  }
  cudaError_t upload(int slot, size_t n, cudaStream_t s) {
    cudaError_t r = cudaMemcpyAsync(dev + (size_t)slot * bytes, host + (size_t)slot * bytes, n,
                                    cudaMemcpyHostToDevice, s);
    if (r != cudaSuccess) return r;
    used[slot] = true;
    return cudaEventRecord(ev[slot], s);
  }
};

class SimBase {
 public:
  virtual ~SimBase() = default;
  std::string err;
  cudaStream_t stream = nullptr;
  virtual void set_state(const double* x0, const double* v0) = 0;
  virtual void set_targets(const double* tv, const double* th, const double* tc) = 0;
  virtual void set_weights(int r, int l, const double* W, const double* b) = 0;
  virtual void get_weights(int r, int l, double* W, double* b) = 0;
  virtual void get_grads(int r, int l, double* gW, double* gb) = 0;
  virtual void forward(int steps, bool eval, bool per_env) = 0;
  virtual void loss(double* terms, double* env) = 0;
  virtual void backward(bool per_env) = 0;
  virtual void adam(int iter, double* tns) = 0;
  virtual void clear_adam() = 0;
  virtual void observables(double* c, double* h, double* u, double* rot) = 0;
  virtual void trajectory(double* x) = 0;
  virtual void targets(double* tv, double* th, double* tc) = 0;
  virtual void set_loss_mask(int mask) = 0;
  virtual void set_loss_envs(int r, int n) = 0;
  virtual void debug_gemm_starve(int starve, unsigned wait_limit) = 0;
  virtual void env_step(int t, const double* outputs, double* obs, double* aux) = 0;
  virtual void env_set_targets(int ue, int t_from, const double* tv, const double* th, const double* tc) = 0;
  virtual void grad_buffers(void** w, long long* nw, void** b, long long* nb, int* elem) = 0;
  virtual void final_state(double* x, double* v) = 0;
  virtual void state_grads(double* gx, double* gv) = 0;
  virtual int synchronize() = 0;
  virtual void graph_capture(int steps, bool with_adam) = 0;
  virtual void graph_launch(int iter) = 0;
  virtual void weights_init(unsigned long long seed) = 0;
  virtual void initialize_train(int iter, int steps, unsigned long long seed, double max_speed) = 0;
  virtual void profile_enable(bool on) = 0;
  virtual void profile_read(double* ms, long long* launches, bool reset) = 0;
  virtual void sizes(int* ne, int* nv, int* T) const = 0;
  virtual void phase_read(unsigned long long* out) = 0;
  virtual void layer_shape(int r, int l, int* rows, int* cols) const = 0;
  // serving: per-env windows over envs at different episode times
  virtual void serve_reset_env(int ue, const double* x0, const double* v0, const double* tv,
                               const double* th, const double* tc) = 0;
  virtual void serve_forward(const int* win, const int* steps) = 0;
  virtual void serve_backward(const int* win, const int* steps) = 0;
  virtual void serve_loss(const int* steps, double* env) = 0;
  virtual void serve_env_state(int ue, double* x, double* v) = 0;
  // what the slot scheduler needs of env ue: its robot class (envs whose
  // robot entries have the same geometry and controller shape share one),
  // vertex count, rest pose and the footprint of a request on it
  virtual int env_class(int ue) const = 0;
  virtual int env_vertices(int ue) const = 0;
  virtual bool env_own_robot(int ue) const = 0;
  virtual const double* env_objects(int ue) const = 0;
  virtual long long env_footprint(int ue, int steps, bool grad) const = 0;
  virtual int checkpoint_every() const = 0;
  // controller path: 0 auto, 1 per env (fused segment kernels), 2 batched
  virtual void set_controller_path(int path) = 0;
  virtual bool controller_batched() const = 0;
  // fused kernels' launch shape and the autotuner over it
  virtual void set_launch_shape(int threads, int ctas, int wsh) = 0;
  virtual void launch_shape(int* threads, int* ctas, int* wsh) const = 0;
  virtual void autotune(int steps, int repeats, std::vector<cls_launch_shape>& table) = 0;
  virtual void set_spring_tables(int mode) = 0;
  virtual bool spring_tables() const = 0;
};

template <typename R>
class SimImpl final : public SimBase {
 public:
  SimImpl(const std::vector<HostRobot>& robots, const std::vector<int>& env_robot,
          const cls_sim_params& p)
      : hr_(robots), p_(p) {
    build(env_robot);
    set_controller_path(0);
  }
  ~SimImpl() override {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
  }

  // ---------------------------------------------------------------- build
  void build(const std::vector<int>& env_robot) {
    const int E = (int)env_robot.size();
    const int nr = (int)hr_.size();
    E_ = E;
    T_ = p_.max_steps;
    K_ = std::max(1, p_.checkpoint_every);
    L_ = hr_[0].n_layers;
    // internal order: envs grouped by robot type (stable)
    perm_.resize(E);  // internal -> user
    std::iota(perm_.begin(), perm_.end(), 0);
    std::stable_sort(perm_.begin(), perm_.end(),
                     [&](int a, int b) { return env_robot[a] < env_robot[b]; });
    identity_perm_ = true;
    for (int i = 0; i < E; ++i) identity_perm_ &= (perm_[i] == i);
    // robot descriptors
    std::vector<RobotDesc> rd(nr);
    std::vector<int> inc_ptr;
    std::vector<int4> inc_i, inc_p;
    std::vector<V4<R>> inc_f;
    std::vector<int> spring_out;
    std::vector<int4> spr_ab;  // per spring {a, b, MLP output or -1, 0}
    std::vector<V4<R>> spr_p;  // per spring {rest length, stiffness, actuation coef, 0}
    int smax = 0;
    long long woff = 0, moff = 0, wtoff = 0;
    int boff = 0;
    nmax_ = 0;
    int p0max = 4, dmax = 4, amax = 4, omax = 4;
    m_off_.assign(nr, std::vector<long long>(L_));
    dd_host_.assign(nr, DenseDesc{});
    for (int r = 0; r < nr; ++r) {
      const HostRobot& h = hr_[r];
      RobotDesc& d = rd[r];
      std::memset(&d, 0, sizeof(d));
      d.n_v = h.n_v;
      d.n_s = h.n_s;
      d.n_out = h.n_out;
      d.n_c = h.n_c;
      d.pos_pad = h.pos_pad;
      d.robot_id = h.robot_id;
      d.n_layers = h.n_layers;
      for (int l = 0; l <= L_; ++l) d.width[l] = h.width[l];
      for (int l = 0; l < L_; ++l) {
        d.pitch[l] = round4(h.width[l]);
        d.w_off[l] = woff;
        woff += (long long)d.pitch[l] * h.width[l + 1];
        woff = (woff + 7) & ~7LL;  // keep every row block 32-byte aligned
        d.b_off[l] = boff;
        boff += round4(h.width[l + 1]);
        m_off_[r][l] = moff;
        moff += (long long)h.width[l + 1] * h.full_cols[l];
        DenseDesc& dd = dd_host_[r];
        dd.wt_pitch[l] = round4(h.width[l + 1]);
        dd.wt_off[l] = wtoff;
        wtoff += (long long)dd.wt_pitch[l] * h.width[l];
        wtoff = (wtoff + 7) & ~7LL;
        TransSeg tsg{};
        tsg.w_off = d.w_off[l]; tsg.wt_off = dd.wt_off[l];
        tsg.rows = h.width[l + 1]; tsg.cols = h.width[l]; tsg.pitch = d.pitch[l]; tsg.wt_pitch = dd.wt_pitch[l];
        tsg.tile0 = n_ttiles_;
        n_ttiles_ += ((tsg.rows + 31) / 32) * ((tsg.cols + 31) / 32);
        tsegs_.push_back(tsg);
      }
      {
        const int Lr = h.n_layers;
        wspan_max_ = std::max(wspan_max_, d.w_off[Lr - 1] + (long long)d.pitch[Lr - 1] * h.width[Lr] -
                                              d.w_off[0]);
        bspan_max_ = std::max(bspan_max_, (long long)(d.b_off[Lr - 1] + round4(h.width[Lr]) - d.b_off[0]));
      }
      int rid[4] = {45, 46, 34, 36};
      for (int q = 0; q < 4; ++q) d.rot_idx[q] = rid[q];
      if (h.robot_id == 100) CLS_REQUIRE(h.n_v > 46, "robot_id 100 needs >= 47 vertices");
      CLS_REQUIRE(h.n_v <= 32767 && h.n_out <= 65534, "robot exceeds the packed incidence limits");
      // CSR incidence, springs sorted by endpoint then by spring index
      d.ptr_off = (int)inc_ptr.size();
      d.inc_off = (int)inc_i.size();
      d.spr_off = (int)spring_out.size();
      std::vector<std::vector<int>> per(h.n_v);
      for (int s = 0; s < h.n_s; ++s) {
        per[h.sa[s]].push_back(2 * s);
        per[h.sb[s]].push_back(2 * s + 1);
      }
      int run = 0;
      for (int i = 0; i < h.n_v; ++i) {
        inc_ptr.push_back(run);
        for (int code : per[i]) {
          const int s = code >> 1, side = code & 1;
          int4 ii;
          ii.x = side ? h.sa[s] : h.sb[s];
          ii.y = side;
          ii.z = s;
          ii.w = h.out[s];
          inc_i.push_back(ii);
          V4<R> f;
          f.x = (R)h.len[s];
          f.y = (R)h.stiff[s];
          f.z = (R)h.coef[s];
          f.w = 0;
          inc_f.push_back(f);
          int4 pk;
          pk.x = (int)((unsigned)ii.x | ((unsigned)side << 15) | ((unsigned)(ii.w + 1) << 16));
          float fl = (float)h.len[s], fk = (float)h.stiff[s], fc = (float)h.coef[s];
          std::memcpy(&pk.y, &fl, 4);
          std::memcpy(&pk.z, &fk, 4);
          std::memcpy(&pk.w, &fc, 4);
          inc_p.push_back(pk);
          ++run;
        }
      }
      inc_ptr.push_back(run);
      for (int s = 0; s < h.n_s; ++s) {
        spring_out.push_back(h.out[s]);
        spr_ab.push_back(make_int4(h.sa[s], h.sb[s], h.out[s], 0));
        V4<R> f;
        f.x = (R)h.len[s];  // the incidence records' values, bit for bit
        f.y = (R)h.stiff[s];
        f.z = (R)h.coef[s];
        f.w = 0;
        spr_p.push_back(f);
      }
      smax = std::max(smax, h.n_s);
      nmax_ = std::max(nmax_, h.n_v);
      p0max = std::max(p0max, round4(h.width[0]));
      omax = std::max(omax, round4(h.n_out));
      dmax = std::max(dmax, round4(h.n_out));
      for (int l = 1; l < L_; ++l) dmax = std::max(dmax, round4(h.width[l]));
      amax = std::max(amax, std::max(round4(h.n_out), h.pos_pad));
      for (int l = 1; l < L_; ++l) amax = std::max(amax, round4(h.width[l]));
    }
    // optimiser / packing segment tables (all robots, all layers)
    {
      long long q = 0, qp = 0;
      for (int r = 0; r < nr; ++r) {
        const HostRobot& h = hr_[r];
        for (int l = 0; l < L_; ++l) {
          OptSeg o{};
          o.start = q; o.m_off = m_off_[r][l]; o.c_off = rd[r].w_off[l];
          o.rows = h.width[l + 1]; o.cols = h.full_cols[l]; o.pitch = rd[r].pitch[l];
          o.layer = l; o.n_v = h.n_v; o.pos_pad = h.pos_pad;
          opt_segs_.push_back(o);
          q += (long long)o.rows * o.cols;
          OptSeg pk = o;
          pk.start = qp;
          pack_segs_.push_back(pk);
          qp += (long long)o.rows * o.pitch;
        }
      }
      for (int r = 0; r < nr; ++r) {
        for (int l = 0; l < L_; ++l) {
          OptSeg o{};
          o.start = q; o.m_off = rd[r].b_off[l]; o.c_off = rd[r].b_off[l];
          o.rows = hr_[r].width[l + 1]; o.cols = 1; o.pitch = 1; o.layer = -1;
          opt_segs_.push_back(o);
          q += o.rows;
        }
      }
      opt_total_ = q;
      pack_total_ = qp;
    }
    // env descriptors (internal order)
    std::vector<EnvDesc> ed(E);
    int voff = 0, inoff = 0;
    int zoff[kMaxLayers] = {0};
    std::vector<int> count(nr, 0), first(nr, -1);
    for (int ie = 0; ie < E; ++ie) {
      const int r = env_robot[perm_[ie]];
      EnvDesc& d = ed[ie];
      std::memset(&d, 0, sizeof(d));
      d.robot = r;
      d.v_off = voff;
      voff += hr_[r].n_v;
      // per-env rows padded to 16 bytes (the batched controller's GEMMs read
      // them as float4)
      d.in_off = inoff;
      inoff += round4(hr_[r].n_c);
      for (int l = 0; l < L_; ++l) {
        d.z_off[l] = zoff[l];
        zoff[l] += round4(hr_[r].width[l + 1]);
      }
      if (first[r] < 0) first[r] = ie;
      count[r]++;
    }
    for (int r = 0; r < nr; ++r) {
      rd[r].n_env = count[r];
      rd[r].loss_envs = count[r];
      rd[r].env_first = first[r] < 0 ? 0 : first[r];
    }
    user_voff_.assign(E, 0);
    {
      std::vector<int> nv_user(E);
      for (int ue = 0; ue < E; ++ue) nv_user[ue] = hr_[env_robot[ue]].n_v;
      int run = 0;
      for (int ue = 0; ue < E; ++ue) { user_voff_[ue] = run; run += nv_user[ue]; }
    }
    env_robot_ = env_robot;
    ed_host_ = ed;
    rd_host_ = rd;
    V_ = voff;
    in_total_ = inoff;
    for (int l = 0; l < L_; ++l) z_total_[l] = zoff[l];
    // controller records: K slots (one segment) or, for episodes of several
    // segments, one slot per substep of the longest episode (slot = t), so
    // that backward() runs the weight-gradient products once over all
    // substeps instead of once per segment.  Whole-episode slots only when no
    // robot type takes the batched controller by default and they need at
    // most a quarter of the free device memory.
    rec_slots_ = K_;
    {
      bool auto_dense = true;
      for (int r = 0; r < nr; ++r)
        if (count[r] > 0 && count[r] < kAutoDenseEnvs) auto_dense = false;
      long long per_slot = in_total_;
      for (int l = 0; l < L_; ++l) per_slot += 2LL * z_total_[l];
      const long long slots_all = std::max(K_, T_ - 1);
      size_t free_b = 0, total_b = 0;
      CLS_CUDA(cudaMemGetInfo(&free_b, &total_b));
      if (T_ - 1 > K_ && !auto_dense &&
          (double)(slots_all - K_) * per_slot * sizeof(R) <= 0.25 * (double)free_b)
        rec_slots_ = (int)slots_all;
    }
    long long zb = 0;
    for (int l = 0; l < L_; ++l) {
      z_base_[l] = zb;
      zb += (long long)rec_slots_ * z_total_[l];
    }
    rec_z_total_ = zb;
    // processing order: heaviest envs first (longest-processing-time first)
    order_host_.resize(E);
    std::iota(order_host_.begin(), order_host_.end(), 0);
    auto cost = [&](int ie) {
      const HostRobot& h = hr_[ed[ie].robot];
      double c = 0;
      for (int l = 0; l < L_; ++l) c += (double)h.width[l + 1] * round4(h.width[l]);
      return c + 40.0 * h.n_s + 20.0 * h.n_v;
    };
    std::stable_sort(order_host_.begin(), order_host_.end(),
                     [&](int a, int b) { return cost(a) > cost(b); });
    // launch shape
    smem_p0max_ = p0max;
    smem_dmax_ = dmax;
    smem_amax_ = amax;
    smem_omax_ = omax;
    // spring impulses computed once per spring into shared memory when the
    // largest robot's table is small (the forward gathers then read them)
    smax_ = smax;
    imp_cap_ = (size_t)smax * sizeof(V4<R>) <= kImpSmemMax ? smax : 0;
    fwd_base_ = fwd_smem_bytes<R>(nmax_, dmax, p0max, imp_cap_);
    int dev = 0;
    CLS_CUDA(cudaGetDevice(&dev));
    CLS_CUDA(cudaDeviceGetAttribute(&n_sm_, cudaDevAttrMultiProcessorCount, dev));
    use_shape(p_.threads_per_block > 0 ? p_.threads_per_block : auto_threads(), -1);
    // GEMM tiles (per robot, per layer); a robot shared by many envs splits
    // its K = envs x substeps rows over several CTAs (about 2048 rows each)
    for (int pass = 0; pass < (rec_slots_ > K_ ? 2 : 1); ++pass) {
      // pass 0: tiles over one segment's rows; pass 1: over the whole episode
      std::vector<GemmTile>& tl = pass ? tiles_ep_ : tiles_host_;
      for (int r = 0; r < nr; ++r) {
        if (count[r] == 0) continue;
        const long long rows = (long long)(pass ? rec_slots_ : K_) * count[r];
        const int nsplit = (int)std::max<long long>(1, std::min<long long>(64, rows / 2048));
        for (int l = 0; l < L_; ++l)
          for (int i0 = 0; i0 < hr_[r].width[l + 1]; i0 += 64)
            for (int j0 = 0; j0 < hr_[r].width[l]; j0 += 64)
              for (int sp = 0; sp < nsplit; ++sp) tl.push_back({r, l, i0, j0, sp, nsplit});
      }
    }
    // device allocations
    const int n_seg_max = (T_ - 1 + K_ - 1) / K_ + 1;
    n_ckpt_ = n_seg_max + 1;
    d_robots_.alloc(nr);
    d_envs_.alloc(E);
    d_order_.alloc(E);
    d_inc_ptr_.alloc(inc_ptr.size());
    d_inc_i_.alloc(std::max<size_t>(1, inc_i.size()));
    d_inc_f_.alloc(std::max<size_t>(1, inc_f.size()));
    d_inc_p_.alloc(std::max<size_t>(1, inc_p.size()));
    d_spring_out_.alloc(std::max<size_t>(1, spring_out.size()));
    d_spr_ab_.alloc(std::max<size_t>(1, spr_ab.size()));
    d_spr_p_.alloc(std::max<size_t>(1, spr_p.size()));
    d_w_.alloc(woff);
    d_gw_.alloc(woff);
    wt_total_ = wtoff;
    d_bias_.alloc(boff);
    d_gb_.alloc(boff);
    d_bm_.alloc(boff);
    d_bv_.alloc(boff);
    d_wm_.alloc(moff);
    d_wmm_.alloc(moff);
    d_wmv_.alloc(moff);
    d_sin_.alloc((size_t)(T_ + 2) * std::max(1, p_.n_sin_waves));
    d_ckx_.alloc((size_t)n_ckpt_ * V_);
    d_ckv_.alloc((size_t)n_ckpt_ * V_);
    d_finx_.alloc(V_);
    d_finv_.alloc(V_);
    d_recx_.alloc((size_t)K_ * V_);
    d_recv_.alloc((size_t)K_ * V_);
    d_recvinc_.alloc((size_t)K_ * V_);
    d_recin_.alloc((size_t)rec_slots_ * in_total_);
    d_recz_.alloc(rec_z_total_);
    d_recdz_.alloc(rec_z_total_);
    d_head_.alloc(V_);
    d_obsc_.alloc((size_t)T_ * E);
    d_obsh_.alloc((size_t)T_ * E);
    d_obsu_.alloc((size_t)T_ * E);
    d_obsr_.alloc((size_t)T_ * E);
    keep_x_ = (p_.loss_mask & (LOSS_ROTATION | LOSS_POSE)) != 0 || p_.keep_trajectory != 0;
    if (keep_x_) d_xfull_.alloc((size_t)T_ * V_);
    if (p_.loss_mask & LOSS_ACTUATION) d_actfull_.alloc((size_t)T_ * z_total_[L_ - 1]);
    d_tv_.alloc((size_t)T_ * E);
    d_th_.alloc((size_t)T_ * E);
    d_tc_.alloc((size_t)T_ * E);
    d_init_.alloc(V_);
    d_adjx_.alloc(V_);
    d_adjv_.alloc(V_);
    d_adjh_.alloc(E);
    d_status_.alloc(1);
#ifdef CLS_PHASE_TIMERS
    d_phase_.alloc(32);
    CLS_CUDA(cudaMemset(d_phase_.p, 0, sizeof(unsigned long long) * 32));
#endif
    d_iter_.alloc(1);
    d_lossenv_.alloc((size_t)E * 8);
    d_tiles_.alloc(std::max<size_t>(1, tiles_host_.size()));
    d_tiles_ep_.alloc(std::max<size_t>(1, tiles_ep_.size()));
    d_opt_segs_.alloc(opt_segs_.size());
    d_pack_segs_.alloc(pack_segs_.size());
    CLS_CUDA(cudaMemcpy(d_opt_segs_.p, opt_segs_.data(), sizeof(OptSeg) * opt_segs_.size(),
                        cudaMemcpyHostToDevice));
    CLS_CUDA(cudaMemcpy(d_pack_segs_.p, pack_segs_.data(), sizeof(OptSeg) * pack_segs_.size(),
                        cudaMemcpyHostToDevice));
    n_queue_ = (size_t)(1 + 2 * n_seg_max) * E;
    d_queue_.alloc(n_queue_);
    d_env_steps_.alloc(E);
    d_sorder_.alloc(E);
    d_squeue_.alloc(2);
    inv_perm_.assign(E, 0);
    for (int ie = 0; ie < E; ++ie) inv_perm_[perm_[ie]] = ie;
    size_t stage = std::max<size_t>((size_t)T_ * E * 3, (size_t)V_ * 3);
    stage = std::max<size_t>(stage, (size_t)moff);
    stage = std::max<size_t>(stage, (size_t)boff);
    d_stage_.alloc(stage);
    d_tns_.alloc(1);
    // uploads
    CLS_CUDA(cudaMemcpy(d_robots_.p, rd.data(), sizeof(RobotDesc) * nr, cudaMemcpyHostToDevice));
    CLS_CUDA(cudaMemcpy(d_envs_.p, ed.data(), sizeof(EnvDesc) * E, cudaMemcpyHostToDevice));
    CLS_CUDA(cudaMemcpy(d_order_.p, order_host_.data(), sizeof(int) * E, cudaMemcpyHostToDevice));
    CLS_CUDA(cudaMemcpy(d_inc_ptr_.p, inc_ptr.data(), sizeof(int) * inc_ptr.size(), cudaMemcpyHostToDevice));
    if (!inc_i.empty()) {
      CLS_CUDA(cudaMemcpy(d_inc_i_.p, inc_i.data(), sizeof(int4) * inc_i.size(), cudaMemcpyHostToDevice));
      CLS_CUDA(cudaMemcpy(d_inc_f_.p, inc_f.data(), sizeof(V4<R>) * inc_f.size(), cudaMemcpyHostToDevice));
      CLS_CUDA(cudaMemcpy(d_inc_p_.p, inc_p.data(), sizeof(int4) * inc_p.size(), cudaMemcpyHostToDevice));
    }
    if (!spr_ab.empty()) {
      CLS_CUDA(cudaMemcpy(d_spr_ab_.p, spr_ab.data(), sizeof(int4) * spr_ab.size(), cudaMemcpyHostToDevice));
      CLS_CUDA(cudaMemcpy(d_spr_p_.p, spr_p.data(), sizeof(V4<R>) * spr_p.size(), cudaMemcpyHostToDevice));
    }
    if (!spring_out.empty()) {
      CLS_CUDA(cudaMemcpy(d_spring_out_.p, spring_out.data(), sizeof(int) * spring_out.size(),
                          cudaMemcpyHostToDevice));
    }
    if (!tiles_ep_.empty())
      CLS_CUDA(cudaMemcpy(d_tiles_ep_.p, tiles_ep_.data(), sizeof(GemmTile) * tiles_ep_.size(),
                          cudaMemcpyHostToDevice));
    if (!tiles_host_.empty())
      CLS_CUDA(cudaMemcpy(d_tiles_.p, tiles_host_.data(), sizeof(GemmTile) * tiles_host_.size(),
                          cudaMemcpyHostToDevice));
    {
      const int ns = std::max(1, p_.n_sin_waves);
      std::vector<R> st((size_t)(T_ + 2) * ns, R(0));
      for (int t = 0; t < T_ + 2; ++t)
        for (int j = 0; j < p_.n_sin_waves; ++j)
          st[(size_t)t * ns + j] =
              (R)std::sin(p_.spring_omega * (double)t * p_.dt + 2 * M_PI / p_.n_sin_waves * (double)j);
      CLS_CUDA(cudaMemcpy(d_sin_.p, st.data(), sizeof(R) * st.size(), cudaMemcpyHostToDevice));
    }
    CLS_CUDA(cudaMemset(d_w_.p, 0, sizeof(R) * d_w_.n));
    CLS_CUDA(cudaMemset(d_wm_.p, 0, sizeof(R) * d_wm_.n));
    CLS_CUDA(cudaMemset(d_bias_.p, 0, sizeof(R) * d_bias_.n));
    CLS_CUDA(cudaMemset(d_ckx_.p, 0, sizeof(V4<R>) * d_ckx_.n));
    CLS_CUDA(cudaMemset(d_ckv_.p, 0, sizeof(V4<R>) * d_ckv_.n));
    CLS_CUDA(cudaMemset(d_tv_.p, 0, sizeof(V4<R>) * d_tv_.n));
    CLS_CUDA(cudaMemset(d_th_.p, 0, sizeof(R) * d_th_.n));
    CLS_CUDA(cudaMemset(d_tc_.p, 0, sizeof(R) * d_tc_.n));
    CLS_CUDA(cudaMemset(d_status_.p, 0, sizeof(int)));
    CLS_CUDA(cudaMemset(d_init_.p, 0, sizeof(V4<R>) * d_init_.n));
    clear_adam();
    // initial state: the robots' own objects
    std::vector<double> x0((size_t)V_ * 3, 0.0);
    for (int ue = 0; ue < E; ++ue) {
      const HostRobot& h = hr_[env_robot[ue]];
      std::memcpy(&x0[(size_t)user_voff_[ue] * 3], h.objects.data(), sizeof(double) * 3 * h.n_v);
    }
    std::vector<double> v0((size_t)V_ * 3, 0.0);
    set_state(x0.data(), v0.data());
    CLS_CUDA(cudaDeviceSynchronize());
  }

  // kernel instances by block size (the register budget follows MAXT)
  using FwdFn = void (*)(MsArgs<R>, int, int, int, int);
  using RevFn = void (*)(MsArgs<R>, int, int, int);
  FwdFn fwd_fn() const {
    return threads_ <= 256 ? ms_forward_kernel<R, 256>
                           : (threads_ <= 512 ? ms_forward_kernel<R, 512> : ms_forward_kernel<R, 1024>);
  }
  RevFn rev_fn() const {
    return threads_ <= 256 ? ms_reverse_kernel<R, 256>
                           : (threads_ <= 512 ? ms_reverse_kernel<R, 512> : ms_reverse_kernel<R, 1024>);
  }

  // Launch shape of the fused kernels: threads per CTA select the kernel
  // instance; its dynamic shared-memory limit is raised, the largest robot
  // must fit and at least one CTA must be resident.  wsh: the controller
  // (weights, biases) in shared memory for a whole work item -- 1 on (it must
  // fit), 0 off (read from global memory every substep), -1 on when it fits
  // without fewer resident CTAs.  The limit is a per-kernel, process-wide
  // attribute: it is raised to the device maximum (minus the kernel's static
  // shared memory) so that handles with different robot sizes never lower it
  // for one another.  On failure the previous shape stays.
  void use_shape(int threads, int wsh) {
    CLS_REQUIRE(threads % 32 == 0 && threads >= 64 && threads <= 1024,
                "threads_per_block must be a multiple of 32 in [64, 1024]");
    CLS_REQUIRE(wsh >= -1 && wsh <= 1, "weights_shared must be -1 (automatic), 0 or 1");
    const int keep = threads_;
    threads_ = threads;
    try {
      const size_t rev0 = rev_smem_bytes<R>(nmax_, smem_amax_, smem_omax_, smem_dmax_, threads, imp_cap_);
      const size_t ctrl = ctrl_smem_bytes<R>(wspan_max_, bspan_max_);
      int dev = 0, optin = 0;
      CLS_CUDA(cudaGetDevice(&dev));
      CLS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
      cudaFuncAttributes fa{}, ra{};
      CLS_CUDA(cudaFuncGetAttributes(&fa, fwd_fn()));
      CLS_CUDA(cudaFuncGetAttributes(&ra, rev_fn()));
      const size_t fwd_cap = (size_t)optin - fa.sharedSizeBytes;
      const size_t rev_cap = (size_t)optin - ra.sharedSizeBytes;
      CLS_REQUIRE(fwd_base_ <= fwd_cap && rev0 <= rev_cap,
                  "robot too large for one CTA's shared memory (" + std::to_string(rev0) +
                      " bytes needed, " + std::to_string(rev_cap) + " available)");
      CLS_CUDA(cudaFuncSetAttribute(fwd_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_cap));
      CLS_CUDA(cudaFuncSetAttribute(rev_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rev_cap));
      // CTAs of both kernels resident per SM with the given shared memory
      auto resident = [&](size_t f, size_t r) {
        if (f > fwd_cap || r > rev_cap) return 0;
        int nf = 0, nb = 0;
        CLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nf, fwd_fn(), threads, f));
        CLS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rev_fn(), threads, r));
        return std::min(nf, nb);
      };
      const int r_off = resident(fwd_base_, rev0);
      CLS_REQUIRE(r_off >= 1,
                  "no CTA of " + std::to_string(threads) + " threads can be resident on an SM");
      const int r_on = resident(fwd_base_ + ctrl, rev0 + ctrl);
      CLS_REQUIRE(wsh != 1 || r_on >= 1,
                  "the controller (" + std::to_string(ctrl) + " bytes) does not fit in shared memory "
                  "beside the kernels' own");
      const bool on = wsh == 1 || (wsh == -1 && r_on >= 1 && r_on >= r_off);
      fwd_smem_ = fwd_base_ + (on ? ctrl : 0);
      rev_smem_ = rev0 + (on ? ctrl : 0);
      resident_ = on ? r_on : r_off;
      wsh_on_ = on;
    } catch (...) {
      threads_ = keep;
      throw;
    }
  }

  // Per-spring tables in shared memory (forward impulses, reverse adjoint
  // terms): -1 when the largest robot's impulse table fits kImpSmemMax (the
  // default), 0 never (direct gathers), 1 on (it must fit).  Recomputes the
  // fused and step kernels' shared memory with the launch shape.
  void set_spring_tables(int mode) override {
    CLS_REQUIRE(!capturing_, "the spring tables cannot change during graph capture");
    CLS_REQUIRE(mode >= -1 && mode <= 1, "spring_tables must be -1 (automatic), 0 or 1");
    const size_t fit = (size_t)smax_ * sizeof(V4<R>) <= kImpSmemMax ? (size_t)smax_ : 0;
    CLS_REQUIRE(mode != 1 || fit, "the spring tables do not fit in shared memory");
    const size_t keep = imp_cap_;
    auto apply = [&](size_t cap) {
      imp_cap_ = cap;
      fwd_base_ = fwd_smem_bytes<R>(nmax_, smem_dmax_, smem_p0max_, imp_cap_);
      use_shape(threads_, wsh_on_ ? 1 : 0);
      if (d_wt_.p) {  // the batched step kernels carve with the same table
        dfwd_smem_ = fwd_smem_bytes<R>(nmax_, smem_omax_, smem_p0max_, imp_cap_);
        int dev = 0, optin = 0;
        CLS_CUDA(cudaGetDevice(&dev));
        CLS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        size_t fwd_static = 0, rev_static = 0;
        CLS_CUDA(DenseLaunch<R>::setup(dense_threads_, &fwd_static, &rev_static, optin));
        CLS_REQUIRE(dfwd_smem_ + fwd_static <= (size_t)optin,
                    "robot too large for the batched controller's step kernels");
      }
    };
    try {
      apply(mode == 0 ? 0 : fit);
    } catch (...) {
      try {
        apply(keep);
      } catch (...) {
      }
      throw;
    }
    fwd_done_ = bwd_done_ = false;
  }
  bool spring_tables() const override { return imp_cap_ > 0; }

  void set_launch_shape(int threads, int ctas, int wsh) override {
    CLS_REQUIRE(!capturing_, "the launch shape cannot change during graph capture");
    CLS_REQUIRE(ctas >= 1 && ctas <= 32, "ctas_per_sm must be in [1, 32]");
    use_shape(threads, wsh);
    ctas_per_sm_ = ctas;
  }
  void launch_shape(int* threads, int* ctas, int* wsh) const override {
    *threads = threads_;
    *ctas = ctas_per_sm_;
    *wsh = wsh_on_ ? 1 : 0;
  }

  // one training rollout (forward, loss, reverse) as the autotuner times it:
  // one untimed run, then `repeats` runs between CUDA events on the stream
  float time_rollout(int steps, int repeats) {
    struct Events {
      cudaEvent_t a = nullptr, b = nullptr;
      ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
      }
    } ev;
    CLS_CUDA(cudaEventCreate(&ev.a));
    CLS_CUDA(cudaEventCreate(&ev.b));
    auto run = [&] {
      forward(steps, false, false);
      loss_device();
      backward(false);
    };
    run();
    CLS_CUDA(cudaEventRecord(ev.a, stream));
    for (int i = 0; i < repeats; ++i) run();
    CLS_CUDA(cudaEventRecord(ev.b, stream));
    CLS_CUDA(cudaEventSynchronize(ev.b));
    float ms = 0;
    CLS_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
    // a timed-out tensor-core wait fails the tuning; non-finite states (the
    // caller's data) do not change the timing and stay for the caller's run
    if (synchronize() == CLS_ERR_CUDA) throw Fail{CLS_ERR_CUDA, err};
    return ms / repeats;
  }

  static constexpr int kTuneDenseEnvs = 32;
  static constexpr int kTuneMaxCtas = 4;

  void autotune(int steps, int repeats, std::vector<cls_launch_shape>& table) override {
    CLS_REQUIRE(!capturing_ && !prof_.on, "autotune needs profiling off and no graph capture");
    if (steps <= 0) steps = std::min(T_, std::min(2 * K_ + 1, 101));
    CLS_REQUIRE(steps >= 2 && steps <= T_, "tuning rollout needs 2 <= steps <= max_steps");
    repeats = std::max(1, repeats);
    const int keep_threads = threads_, keep_ctas = ctas_per_sm_, keep_wsh = wsh_on_ ? 1 : 0;
    const bool keep_dense = dense_;
    bool can_dense = true;
    for (const RobotDesc& d : rd_host_)
      if (d.n_env > 0 && d.n_env < kTuneDenseEnvs) can_dense = false;
    table.clear();
    try {
      dense_ = false;
      for (int threads : {128, 256, 512, 1024}) {
        for (int wsh : {0, 1}) {
          try {
            use_shape(threads, wsh);
          } catch (const Fail& f) {
            if (f.code != CLS_ERR_INVALID) throw;
            continue;  // the largest robot (or its controller) does not fit this instance
          }
          for (int ctas = 1; ctas <= std::min(resident_, kTuneMaxCtas); ++ctas) {
            ctas_per_sm_ = ctas;
            table.push_back({CLS_CONTROLLER_PER_ENV, threads, ctas, wsh, time_rollout(steps, repeats)});
          }
        }
      }
      CLS_REQUIRE(!table.empty(), "no launch shape fits the largest robot");
      size_t best = 0;
      for (size_t i = 1; i < table.size(); ++i)
        if (table[i].ms < table[best].ms) best = i;
      // the fused kernels keep their fastest shape (per-env launches and
      // serving windows use them on either controller path)
      use_shape(table[best].threads_per_block, table[best].weights_shared);
      ctas_per_sm_ = table[best].ctas_per_sm;
      if (can_dense) {
        set_controller_path(CLS_CONTROLLER_BATCHED);
        table.push_back({CLS_CONTROLLER_BATCHED, threads_, ctas_per_sm_, wsh_on_ ? 1 : 0,
                         time_rollout(steps, repeats)});
        if (table.back().ms >= table[best].ms) set_controller_path(CLS_CONTROLLER_PER_ENV);
      } else {
        set_controller_path(CLS_CONTROLLER_PER_ENV);
      }
    } catch (...) {
      try {
        use_shape(keep_threads, keep_wsh);
      } catch (...) {
      }
      ctas_per_sm_ = keep_ctas;
      dense_ = keep_dense;
      fwd_done_ = bwd_done_ = false;
      throw;
    }
  }

  int auto_threads() const {
    // enough warps for the per-row MLP products and the vertex loops; more
    // threads than that only adds barrier cost
    int work = 0;
    for (const HostRobot& h : hr_) {
      work = std::max(work, h.n_v);
      for (int l = 1; l <= L_; ++l) work = std::max(work, h.width[l] * 4);
    }
    int t = 128;
    while (t < 512 && t < work) t *= 2;
    return t;
  }

  MsArgs<R> args(int steps) const {
    MsArgs<R> a;
    std::memset(&a, 0, sizeof(a));
    a.n_envs = E_;
    a.n_items = E_;
    a.T = T_;
    a.steps = steps;
    a.K = K_;
    a.n_sin = p_.n_sin_waves;
    a.dup_v = p_.duplicate_v;
    a.dup_h = p_.duplicate_h;
    a.dup_c = p_.duplicate_c;
    a.act_hidden = p_.activation_hidden;
    a.act_out = p_.activation_output;
    a.run_period = p_.run_period;
    a.turn_period = p_.turn_period;
    a.jump_period = p_.jump_period;
    a.loss_mask = p_.loss_mask;
    a.v_total = V_;
    a.in_total = in_total_;
    for (int l = 0; l < L_; ++l) {
      a.z_total[l] = z_total_[l];
      a.z_base[l] = z_base_[l];
    }
    a.smem_nmax = nmax_;
    a.smem_p0max = smem_p0max_;
    a.smem_dmax = smem_dmax_;
    a.smem_amax = smem_amax_;
    a.smem_omax = smem_omax_;
    a.w_smem = wsh_on_ ? (int)wspan_max_ : 0;
    a.b_smem = wsh_on_ ? (int)bspan_max_ : 0;
    a.dt = (R)p_.dt;
    a.gravity = (R)p_.gravity;
    a.ground = (R)p_.ground_height;
    a.drag_s = (R)std::exp(-p_.dt * p_.drag_damping);
    a.dashpot = (R)p_.dashpot_damping;
    a.friction = (R)p_.friction;
    a.max_speed = (R)p_.max_speed;
    a.robots = d_robots_.p;
    a.envs = d_envs_.p;
    a.order = d_order_.p;
    a.queue = d_queue_.p;
    a.inc_ptr = d_inc_ptr_.p;
    a.inc_i = d_inc_i_.p;
    a.inc_f = d_inc_f_.p;
    a.inc_p = d_inc_p_.p;
    a.spring_out = d_spring_out_.p;
    a.spr_ab = d_spr_ab_.p;
    a.spr_p = d_spr_p_.p;
    a.imp_cap = (int)imp_cap_;
    a.adj_cap = (int)imp_cap_;
    a.w = d_w_.p;
    a.bias = d_bias_.p;
    a.sin_table = d_sin_.p;
    a.ckpt_x = d_ckx_.p;
    a.ckpt_v = d_ckv_.p;
    a.fin_x = d_finx_.p;
    a.fin_v = d_finv_.p;
    a.rec_x = d_recx_.p;
    a.rec_v = d_recv_.p;
    a.rec_vinc = d_recvinc_.p;
    a.rec_in = d_recin_.p;
    a.rec_z = d_recz_.p;
    a.rec_dz = d_recdz_.p;
    a.head = d_head_.p;
    a.obs_center = d_obsc_.p;
    a.obs_height = d_obsh_.p;
    a.obs_upper = d_obsu_.p;
    a.obs_rot = d_obsr_.p;
    a.x_full = d_xfull_.p;
    a.act_full = d_actfull_.p;
    a.tv = d_tv_.p;
    a.th = d_th_.p;
    a.tc = d_tc_.p;
    a.init_obj = d_init_.p;
    a.adj_x = d_adjx_.p;
    a.adj_v = d_adjv_.p;
    a.adj_h = d_adjh_.p;
    a.status = d_status_.p;
    a.gemm_wait_limit = gemm_wait_limit_;
    a.gemm_starve = gemm_starve_;
    a.phase = d_phase_.p;
    a.live_x = d_livex_.p;
    a.live_v = d_livev_.p;
    a.din = d_din_.p;
    a.wt = d_wt_.p;
    a.tiles = d_split_.p;
    a.dense = d_dense_.p;
    a.wtiles = d_wsplit_.p;
    return a;
  }

  int grid_for(int items) const { return std::max(1, std::min(items, n_sm_ * ctas_per_sm_)); }

  // one batched launch (all envs) or one launch per env
  template <typename F>
  void each_launch(bool per_env, MsArgs<R> a, int& qslot, F&& launch) {
    if (!per_env) {
      a.queue = d_queue_.p + (size_t)qslot * 1;
      qslot += 1;
      launch(a, grid_for(E_));
      return;
    }
    for (int k = 0; k < E_; ++k) {
      MsArgs<R> b = a;
      b.order = d_order_.p + k;
      b.n_items = 1;
      b.queue = d_queue_.p + (size_t)qslot;
      qslot += 1;
      launch(b, 1);
    }
  }

  // run one kernel launch, counted and (when profiling) bracketed by events
  template <typename F>
  void timed(int kind, F&& f) {
    CLS_CUDA(prof_.run(kind, stream, std::forward<F>(f)));
  }

  void profile_collect() { CLS_CUDA(prof_.collect(stream)); }

  void profile_enable(bool on) override {
    CLS_REQUIRE(!capturing_, "profiling cannot be switched during graph capture");
    profile_collect();
    prof_.on = on;
  }

  void profile_read(double* ms, long long* launches, bool reset) override {
    profile_collect();
    prof_.read(ms, launches, reset);
  }

  void weights_init(unsigned long long seed) override {
    const int chunk = 256 * 16;
    const int blocks = (int)((opt_total_ + chunk - 1) / chunk);
    timed(PK_OTHER, [&] {
      ms_weights_init_all_kernel<R><<<std::max(1, blocks), 256, 0, stream>>>(
          d_opt_segs_.p, (int)opt_segs_.size(), opt_total_, chunk, d_wm_.p, seed);
    });
    pack_all();
    CLS_CUDA(cudaGetLastError());
  }

  void initialize_train(int iter, int steps, unsigned long long seed, double max_speed) override {
    CLS_REQUIRE(steps >= 1 && steps <= T_, "steps out of range");
    const long long n = (long long)T_ * E_;
    // the sampled tasks are defined per internal env; targets of envs are
    // independent draws, so the env numbering only relabels the draws
    timed(PK_OTHER, [&] {
      ms_initialize_train_kernel<R><<<blocks_for(n), 256, 0, stream>>>(
          d_tv_.p, d_th_.p, T_, steps, E_, p_.turn_period, seed, iter, max_speed);
    });
    CLS_CUDA(cudaGetLastError());
  }

  // --------------------------------------------------------------- passes
  void forward(int steps, bool eval, bool per_env) override {
    if (eval) {
      CLS_REQUIRE(steps >= 0 && steps + 1 < T_, "evaluation rollout needs steps + 1 < max_steps");
    } else {
      CLS_REQUIRE(steps >= 2 && steps <= T_, "training rollout needs 2 <= steps <= max_steps");
    }
    steps_ = steps;
    eval_ = eval;
    per_env_ = per_env;
    CLS_CUDA(cudaMemsetAsync(d_queue_.p, 0, sizeof(int) * d_queue_.n, stream));
    CLS_CUDA(cudaMemsetAsync(d_obsc_.p, 0, sizeof(V4<R>) * d_obsc_.n, stream));
    CLS_CUDA(cudaMemsetAsync(d_obsh_.p, 0, sizeof(R) * d_obsh_.n, stream));
    CLS_CUDA(cudaMemsetAsync(d_obsu_.p, 0, sizeof(R) * d_obsu_.n, stream));
    CLS_CUDA(cudaMemsetAsync(d_obsr_.p, 0, sizeof(R) * d_obsr_.n, stream));
    if (d_xfull_.p) CLS_CUDA(cudaMemsetAsync(d_xfull_.p, 0, sizeof(V4<R>) * d_xfull_.n, stream));
    if (d_actfull_.p) CLS_CUDA(cudaMemsetAsync(d_actfull_.p, 0, sizeof(R) * d_actfull_.n, stream));
    const int t_end = eval ? steps + 1 : steps - 1;
    MsArgs<R> a = args(steps);
    qslot_ = 0;
    // a training episode of one checkpoint segment (steps - 1 <= K): the first
    // pass records what the segment's recompute would (same kernels, same
    // values), and the reverse pass starts without a recompute
    recorded_ = !eval && t_end <= K_;
    int mode = FWD_CKPT | FWD_OBS | (recorded_ ? FWD_RECORD : 0);
    // An episode of several segments run by the fused kernels: the first
    // pass also records the last segment (FWD_RECTAIL) where that segment's
    // recompute would, and the reverse pass skips that recompute.  With
    // whole-episode controller records it also records every substep's
    // controller at slot t (FWD_RECCTRL), and the reverse pass's recomputes
    // replay the controller outputs from those records (FWD_REPLAY) instead
    // of evaluating the controller again.
    tail_recorded_ = false;
    tail_episode_ = false;
    if (!eval && t_end > K_ && (!dense_ || per_env)) {
      const int n_seg = (t_end + K_ - 1) / K_;
      a.rec_from = (n_seg - 1) * K_;
      tail_episode_ = episode_records();
      mode |= FWD_RECTAIL | (tail_episode_ ? FWD_RECCTRL : 0);
      tail_recorded_ = true;
    }
    if (dense_ && !per_env) {
      dense_pass(a, 0, t_end, mode, 0, true, PK_FWD);
    } else {
      each_launch(per_env, a, qslot_, [&](const MsArgs<R>& b, int grid) {
        timed(PK_FWD, [&] { fwd_fn()<<<grid, threads_, fwd_smem_, stream>>>(b, 0, t_end, mode, 0); });
      });
    }
    CLS_CUDA(cudaGetLastError());
    fwd_done_ = true;
  }


  // ------------------------------------------------- batched controller
  // Robot types with at least this many envs take the batched path when the
  // controller path is automatic.
  static constexpr int kAutoDenseEnvs = 256;

  bool controller_batched() const override { return dense_; }

  void set_controller_path(int path) override {
    CLS_REQUIRE(path >= 0 && path <= 2, "controller path: 0 automatic, 1 per env, 2 batched");
    CLS_REQUIRE(!capturing_, "the controller path cannot change during graph capture");
    bool want = path == 2;
    if (path == 0) {
      want = true;
      for (const RobotDesc& d : rd_host_)
        if (d.n_env > 0 && d.n_env < kAutoDenseEnvs) want = false;
    }
    if (want && !d_wt_.p) enable_dense();
    dense_ = want;
    fwd_done_ = bwd_done_ = false;
  }

  void enable_dense() {
    constexpr bool f32 = std::is_same<R, float>::value;
    const int tm = DenseLaunch<R>::tile_m(), tn = DenseLaunch<R>::tile_n();
    jobs_h_.clear();
    for (int l = 0; l < L_; ++l) {
      jf_off_[l] = (int)jobs_h_.size();
      for (int r = 0; r < (int)hr_.size(); ++r) {
        if (rd_host_[r].n_env == 0 || l >= hr_[r].n_layers) continue;
        for (int m0 = 0; m0 < rd_host_[r].n_env; m0 += tm)
          for (int n0 = 0; n0 < hr_[r].width[l + 1]; n0 += tn) jobs_h_.push_back({r, l, m0, n0});
      }
      jf_cnt_[l] = (int)jobs_h_.size() - jf_off_[l];
    }
    for (int l = 0; l < L_; ++l) {
      jb_off_[l] = (int)jobs_h_.size();
      for (int r = 0; r < (int)hr_.size(); ++r) {
        if (rd_host_[r].n_env == 0 || l >= hr_[r].n_layers) continue;
        const int ncol = l > 0 ? hr_[r].width[l] : 3 * hr_[r].n_v;
        for (int m0 = 0; m0 < rd_host_[r].n_env; m0 += tm)
          for (int n0 = 0; n0 < ncol; n0 += tn) jobs_h_.push_back({r, l, m0, n0});
      }
      jb_cnt_[l] = (int)jobs_h_.size() - jb_off_[l];
    }
    d_jobs_.alloc(std::max<size_t>(1, jobs_h_.size()));
    CLS_CUDA(cudaMemcpy(d_jobs_.p, jobs_h_.data(), sizeof(DenseJob) * jobs_h_.size(), cudaMemcpyHostToDevice));
    d_tsegs_.alloc(std::max<size_t>(1, tsegs_.size()));
    CLS_CUDA(cudaMemcpy(d_tsegs_.p, tsegs_.data(), sizeof(TransSeg) * tsegs_.size(), cudaMemcpyHostToDevice));
    d_livex_.alloc(V_);
    d_livev_.alloc(V_);
    d_din_.alloc((size_t)3 * V_);
    d_wt_.alloc(std::max<long long>(1, wt_total_));
    CLS_CUDA(cudaMemset(d_wt_.p, 0, sizeof(R) * d_wt_.n));
    if constexpr (f32) {
      // pre-split operand tiles of every layer's GEMMs (zero padding stays zero)
      long long off = 0;
      ssegs_.clear();
      split_total_ = 0;
      for (int r = 0; r < (int)hr_.size(); ++r) {
        const RobotDesc& d = rd_host_[r];
        DenseDesc& dd = dd_host_[r];
        const HostRobot& h = hr_[r];
        if (d.n_env == 0) continue;
        for (int l = 0; l < h.n_layers; ++l) {
          const int wi = h.width[l], wo = h.width[l + 1];
          dd.ta_f[l] = off; off += DenseLaunch<R>::split_floats(d.n_env, tm, wi);
          dd.ta_b[l] = off; off += DenseLaunch<R>::split_floats(d.n_env, tm, wo);
          dd.tb_f[l] = off; off += DenseLaunch<R>::split_floats(wo, tn, wi);
          dd.tb_b[l] = off; off += DenseLaunch<R>::split_floats(wi, tn, wo);
          SplitSeg sg{};
          sg.w_off = d.w_off[l]; sg.tf_off = dd.tb_f[l]; sg.tb_off = dd.tb_b[l];
          sg.rows = wo; sg.cols = wi; sg.pitch = d.pitch[l]; sg.first = split_total_;
          split_total_ += (long long)wo * wi;
          ssegs_.push_back(sg);
        }
      }
      d_split_.alloc(std::max<long long>(1, off));
      CLS_CUDA(cudaMemset(d_split_.p, 0, sizeof(R) * d_split_.n));
      // weight-gradient operands of one segment (K = record slots x envs
      // padded to 32) and the per-segment transpose / tile lists
      long long woff = 0;
      wg_trans_.clear(); wg_cols_.clear(); wg_jobs_.clear();
      wg_grid_x_ = 0;
      wg_chunk_ = std::min(K_, kWgChunkSlots);
      int n_tiles = 0;
      for (int r = 0; r < (int)hr_.size(); ++r) {
        const RobotDesc& d = rd_host_[r];
        DenseDesc& dd = dd_host_[r];
        const HostRobot& h = hr_[r];
        if (d.n_env == 0) continue;
        dd.nep = (d.n_env + 31) & ~31;
        dd.nkt_w = wg_chunk_ * dd.nep / 32;
        wg_grid_x_ = std::max(wg_grid_x_, dd.nep / 32);
        for (int l = 0; l < h.n_layers; ++l) {
          const int wi = h.width[l], wo = h.width[l + 1];
          dd.tw_d[l] = woff; woff += DenseLaunch<R>::split_floats(wo, tm, wg_chunk_ * dd.nep);
          dd.tw_a[l] = woff; woff += DenseLaunch<R>::split_floats(wi + 1, tn, wg_chunk_ * dd.nep);
          const WgTrans ta{r, l, l == 0 ? 0 : 1, wi}, td{r, l, 2, wo};
          for (const WgTrans& tr : {ta, td}) {
            const int job = (int)wg_trans_.size();
            wg_trans_.push_back(tr);
            const int rows = tr.cols + (tr.kind == 2 ? 0 : 1);
            for (int c0 = 0; c0 < rows; c0 += 32) wg_cols_.push_back({job, c0});
          }
          n_tiles += ((wo + tm - 1) / tm) * ((wi + 1 + tn - 1) / tn);
        }
      }
      // K splits: about two CTAs per SM, at least 8 K blocks each
      int max_kt = 0;
      for (const DenseDesc& dd : dd_host_) max_kt = std::max(max_kt, dd.nkt_w);
      const int nsplit = std::max(1, std::min(std::max(1, max_kt / 8), (2 * n_sm_ + n_tiles - 1) / std::max(1, n_tiles)));
      // split outermost: the tiles of one K range run together and share
      // their operand blocks through L2 (a segment's operands exceed it)
      for (int sp = 0; sp < nsplit; ++sp)
        for (int r = 0; r < (int)hr_.size(); ++r) {
          if (rd_host_[r].n_env == 0) continue;
          const HostRobot& h = hr_[r];
          for (int l = 0; l < h.n_layers; ++l)
            for (int o0 = 0; o0 < h.width[l + 1]; o0 += tm)
              for (int i0 = 0; i0 < h.width[l] + 1; i0 += tn) wg_jobs_.push_back({r, l, o0, i0, sp, nsplit});
        }
      d_wsplit_.alloc(std::max<long long>(1, woff));
      CLS_CUDA(cudaMemset(d_wsplit_.p, 0, sizeof(R) * d_wsplit_.n));
      d_wg_trans_.alloc(std::max<size_t>(1, wg_trans_.size()));
      d_wg_cols_.alloc(std::max<size_t>(1, wg_cols_.size()));
      d_wg_jobs_.alloc(std::max<size_t>(1, wg_jobs_.size()));
      CLS_CUDA(cudaMemcpy(d_wg_trans_.p, wg_trans_.data(), sizeof(WgTrans) * wg_trans_.size(), cudaMemcpyHostToDevice));
      CLS_CUDA(cudaMemcpy(d_wg_cols_.p, wg_cols_.data(), sizeof(WgCol) * wg_cols_.size(), cudaMemcpyHostToDevice));
      CLS_CUDA(cudaMemcpy(d_wg_jobs_.p, wg_jobs_.data(), sizeof(WgJob) * wg_jobs_.size(), cudaMemcpyHostToDevice));
      d_ssegs_.alloc(std::max<size_t>(1, ssegs_.size()));
      CLS_CUDA(cudaMemcpy(d_ssegs_.p, ssegs_.data(), sizeof(SplitSeg) * ssegs_.size(), cudaMemcpyHostToDevice));
    }
    d_dense_.alloc(std::max<size_t>(1, dd_host_.size()));
    CLS_CUDA(cudaMemcpy(d_dense_.p, dd_host_.data(), sizeof(DenseDesc) * dd_host_.size(), cudaMemcpyHostToDevice));
    // step kernels: one CTA of CLS_STEP_THREADS threads per env (64 and 128
    // measured the same on the 4096-env spider); per CTA the fused kernels'
    // shared-memory carve with the controller buffers sized for the output
    // layer only (step_args)
    dense_threads_ = CLS_STEP_THREADS;
    dfwd_smem_ = fwd_smem_bytes<R>(nmax_, smem_omax_, smem_p0max_, imp_cap_);
    drev_smem_ = rev_smem_bytes<R>(nmax_, smem_amax_, smem_omax_, smem_omax_, dense_threads_, 0);
    int dev = 0, optin = 0;
    CLS_CUDA(cudaGetDevice(&dev));
    CLS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    size_t fwd_static = 0, rev_static = 0;
    CLS_CUDA(DenseLaunch<R>::setup(dense_threads_, &fwd_static, &rev_static, optin));
    CLS_REQUIRE(dfwd_smem_ + fwd_static <= (size_t)optin && drev_smem_ + rev_static <= (size_t)optin,
                "robot too large for the batched controller's step kernels");
    transpose_weights();
    CLS_CUDA(cudaStreamSynchronize(stream));
  }

  // launch arguments of the step kernels: the shared-memory carve sizes the
  // controller buffers for the output layer only
  MsArgs<R> step_args(const MsArgs<R>& a) const {
    MsArgs<R> b = a;
    b.smem_dmax = smem_omax_;
    b.w_smem = b.b_smem = 0;  // the step kernels read the controller from its GEMM tiles
    b.adj_cap = 0;            // and keep their residency: the spring adjoint gathers directly
    b.n_items = E_;
    return b;
  }
  int step_grid() const { return E_; }

  // one layer's GEMM over all batched envs (record slot kslot)
  void ctrl_gemm(const MsArgs<R>& a, bool bwd, int l, int kslot) {
    const int cnt = bwd ? jb_cnt_[l] : jf_cnt_[l];
    if (cnt == 0) return;
    const DenseJob* jobs = d_jobs_.p + (bwd ? jb_off_[l] : jf_off_[l]);
    timed(bwd ? PK_CGEMM_ADJ : PK_CGEMM, [&] { DenseLaunch<R>::gemm(a, bwd, cnt, jobs, kslot, stream); });
  }

  // forward over [t_first, t_end): a step launch per substep boundary and the
  // controller's GEMMs in between.  Record slots: t mod K for the first pass
  // (the controller's records are only scratch there), t - t_first for a
  // segment recompute.
  void dense_pass(const MsArgs<R>& a, int t_first, int t_end, int mode, int src_slot, bool first_pass,
                  int kind) {
    for (int t = t_first; t <= t_end; ++t) {
      const int k_prev = t > t_first ? (first_pass ? (t - 1) % K_ : t - 1 - t_first) : 0;
      const int k_cur = t < t_end ? (first_pass ? t % K_ : t - t_first) : 0;
      timed(kind, [&] {
        DenseLaunch<R>::step_fwd(step_args(a), step_grid(), dense_threads_, dfwd_smem_, stream, t, t_first, t_end, mode,
                                 src_slot, k_prev, k_cur);
      });
      if (t < t_end)
        for (int l = 0; l < L_; ++l) ctrl_gemm(a, false, l, k_cur);
    }
  }

  // reverse of segment [t0, t1): step launches from t1 - 1 down to t0 - 1,
  // the controller's adjoint GEMMs after each launch that ends in dZ
  void dense_reverse(const MsArgs<R>& a, int t0, int t1, bool last) {
    for (int t = t1 - 1; t >= t0 - 1; --t) {
      const int t_post = (t + 1 < t1) ? t + 1 : -1;
      const int t_pre = (t >= t0) ? t : -1;
      timed(PK_REV, [&] {
        DenseLaunch<R>::step_rev(step_args(a), step_grid(), dense_threads_, drev_smem_, stream, t_post, t_pre, t0, t1,
                                 last ? 1 : 0);
      });
      if (t_pre >= 0)
        for (int l = L_ - 1; l >= 0; --l) ctrl_gemm(a, true, l, t_pre - t0);
    }
  }

  void loss_device() {
    MsArgs<R> a = args(steps_);
    timed(PK_LOSS, [&] { ms_loss_kernel<R><<<E_, 512, 0, stream>>>(a, d_lossenv_.p, nullptr); });
    CLS_CUDA(cudaGetLastError());
  }

  void loss(double* terms, double* env) override {
    CLS_REQUIRE(fwd_done_, "cls_loss called before a forward rollout");
    loss_device();
    std::vector<double> raw((size_t)E_ * 8);
    CLS_CUDA(cudaMemcpyAsync(raw.data(), d_lossenv_.p, sizeof(double) * raw.size(),
                             cudaMemcpyDeviceToHost, stream));
    CLS_CUDA(cudaStreamSynchronize(stream));
    loss_from_raw(raw, terms, env);
  }

  void loss_from_raw(const std::vector<double>& raw, double* terms, double* env) {
    double t8[8] = {0};
    for (int ie = 0; ie < E_; ++ie)
      for (int l = 0; l < LS_COUNT; ++l) t8[1 + l] += raw[(size_t)ie * 8 + l];
    for (int l = 1; l < 8; ++l) t8[0] += t8[l];
    if (terms) std::memcpy(terms, t8, sizeof(t8));
    if (env) {
      for (int ie = 0; ie < E_; ++ie) {
        const int ue = perm_[ie];
        const double B = rd_host_[ed_host_[ie].robot].loss_envs;
        double tot = 0;
        for (int l = 0; l < LS_COUNT; ++l) {
          const double v = raw[(size_t)ie * 8 + l] * B;
          env[(size_t)(1 + l) * E_ + ue] = v;
          tot += v;
        }
        env[ue] = tot;
      }
    }
    max_height_ = 0;
    for (int ie = 0; ie < E_; ++ie) max_height_ = std::max(max_height_, raw[(size_t)ie * 8 + 7]);
  }

  void backward(bool per_env) override {
    CLS_REQUIRE(fwd_done_ && !eval_, "cls_backward needs a training rollout first");
    const int steps = steps_;
    const int t_last = steps - 1;  // x[steps-1] is the last state
    const int n_seg = (t_last + K_ - 1) / K_;
    CLS_CUDA(cudaMemsetAsync(d_gw_.p, 0, sizeof(R) * d_gw_.n, stream));
    CLS_CUDA(cudaMemsetAsync(d_gb_.p, 0, sizeof(R) * d_gb_.n, stream));
    const MsArgs<R> a0 = args(steps);
    int qslot = qslot_;
    // whole-episode records: segment s's records sit at slots t (the
    // segment's slot kk = t - t0 shifted by t0), and the weight-gradient
    // products run once after the loop over slots [0, t_last)
    const bool episode = episode_records() && (!dense_ || per_env) && n_seg > 1;
    // the first pass recorded the last segment in the layout this pass reads
    const bool tail = tail_recorded_ && (!dense_ || per_env) && n_seg > 1 && tail_episode_ == episode;
    for (int s = n_seg - 1; s >= 0; --s) {
      const int t0 = s * K_, t1 = std::min(t0 + K_, t_last);
      const bool recompute = !(recorded_ && n_seg == 1) && !(tail && s == n_seg - 1);
      MsArgs<R> a = a0;
      if (episode) {
        for (int l = 0; l < L_; ++l) a.z_base[l] += (long long)t0 * z_total_[l];
        a.rec_in += (size_t)t0 * in_total_;
      }
      if (dense_ && !per_env) {
        if (recompute) dense_pass(a, t0, t1, FWD_RECORD, s, false, PK_RECOMP);
        dense_reverse(a, t0, t1, s == n_seg - 1);
      } else {
        // the first pass recorded every substep's controller in this layout:
        // replay its outputs
        const int rmode = FWD_RECORD | (tail && episode ? FWD_REPLAY : 0);
        if (recompute)
          each_launch(per_env, a, qslot, [&](const MsArgs<R>& b, int grid) {
            timed(PK_RECOMP, [&] {
              fwd_fn()<<<grid, threads_, fwd_smem_, stream>>>(b, t0, t1, rmode, s);
            });
          });
        each_launch(per_env, a, qslot, [&](const MsArgs<R>& b, int grid) {
          timed(PK_REV, [&] {
            rev_fn()<<<grid, threads_, rev_smem_, stream>>>(b, t0, t1, s == n_seg - 1 ? 1 : 0);
          });
        });
      }
      if (episode) continue;
      if (dense_ && !per_env && !wg_jobs_.empty()) {
        // FP32 batched path: record transposes + tensor-core tiles, in chunks
        // of at most wg_chunk_ record slots (the operand buffers' size)
        for (int c0 = 0; c0 < t1 - t0; c0 += wg_chunk_) {
          const int c1 = std::min(t1 - t0, c0 + wg_chunk_);
          timed(PK_WGRAD, [&] {
            DenseLaunch<R>::wgrad(a, wg_grid_x_, (int)wg_cols_.size(), c0, c1 - c0, d_wg_trans_.p, d_wg_cols_.p,
                                  (int)wg_jobs_.size(), d_wg_jobs_.p, d_gw_.p, d_gb_.p, stream);
          });
        }
      } else if (!tiles_host_.empty()) {
        timed(PK_WGRAD, [&] {
          ms_wgrad_kernel<R><<<(int)tiles_host_.size(), 256, 0, stream>>>(a, d_tiles_.p, t1 - t0,
                                                                           d_gw_.p, d_gb_.p);
        });
      }
    }
    if (episode)
      timed(PK_WGRAD, [&] {
        ms_wgrad_kernel<R><<<(int)tiles_ep_.size(), 256, 0, stream>>>(a0, d_tiles_ep_.p, t_last, d_gw_.p,
                                                                        d_gb_.p);
      });
    CLS_CUDA(cudaGetLastError());
    bwd_done_ = true;
  }

  void adam_device(int iter_or_neg, bool apply, double* tns_dev) {
    // iteration taken from d_iter_ when iter_or_neg < 0 (graph replays)
    const int chunk = 256 * 16;
    const int blocks = (int)((opt_total_ + chunk - 1) / chunk);
    if (tns_dev) CLS_CUDA(cudaMemsetAsync(tns_dev, 0, sizeof(double), stream));
    timed(PK_ADAM, [&] {
      ms_adam_all_kernel<R><<<std::max(1, blocks), 256, 0, stream>>>(
          d_opt_segs_.p, (int)opt_segs_.size(), opt_total_, chunk, d_wm_.p, d_wmm_.p, d_wmv_.p,
          d_gw_.p, d_bias_.p, d_bm_.p, d_bv_.p, d_gb_.p, p_.n_sin_waves, p_.duplicate_v,
          p_.duplicate_h, p_.duplicate_c, p_.learning_rate, p_.adam_b1, p_.adam_b2, iter_or_neg,
          d_iter_.p, apply ? 1 : 0, tns_dev);
    });
    if (apply) pack_all();
    CLS_CUDA(cudaGetLastError());
  }

  void pack_all() {
    const int chunk = 256 * 16;
    const int blocks = (int)((pack_total_ + chunk - 1) / chunk);
    timed(PK_ADAM, [&] {
      ms_pack_all_kernel<R><<<std::max(1, blocks), 256, 0, stream>>>(
          d_pack_segs_.p, (int)pack_segs_.size(), pack_total_, chunk, d_wm_.p, d_w_.p,
          p_.n_sin_waves, p_.duplicate_v, p_.duplicate_h, p_.duplicate_c);
    });
    transpose_weights();
  }

  // W_l^T of every layer for the batched controller's adjoint GEMMs (only
  // once the batched path has been enabled)
  void transpose_weights() {
    if (!d_wt_.p || n_ttiles_ == 0) return;
    // FP32: the GEMMs read W_l and W_l^T as pre-split tiles; FP64: W_l^T
    timed(PK_ADAM, [&] {
      DenseLaunch<R>::pack_weights(d_w_.p, d_wt_.p, d_split_.p, d_tsegs_.p, (int)tsegs_.size(), n_ttiles_,
                                   d_ssegs_.p, (int)ssegs_.size(), split_total_, stream);
    });
  }

  void adam(int iter, double* tns) override {
    CLS_REQUIRE(bwd_done_, "cls_adam_step needs gradients (cls_backward) first");
    adam_device(iter, true, tns ? d_tns_.p : nullptr);
    if (tns) {
      CLS_CUDA(cudaMemcpyAsync(&tns_host_, d_tns_.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
      *tns = tns_host_;
    }
  }

  void clear_adam() override {
    CLS_CUDA(cudaMemset(d_wmm_.p, 0, sizeof(R) * d_wmm_.n));
    CLS_CUDA(cudaMemset(d_wmv_.p, 0, sizeof(R) * d_wmv_.n));
    CLS_CUDA(cudaMemset(d_bm_.p, 0, sizeof(R) * d_bm_.n));
    CLS_CUDA(cudaMemset(d_bv_.p, 0, sizeof(R) * d_bv_.n));
  }

  void pack_layer(int r, int l) {
    const HostRobot& h = hr_[r];
    const RobotDesc& d = rd_host_[r];
    const long long total = (long long)h.width[l + 1] * d.pitch[l];
    const int blocks = (int)std::min<long long>(1024, (total + 255) / 256);
    timed(PK_ADAM, [&] {
      ms_pack_weights_kernel<R><<<std::max(1, blocks), 256, 0, stream>>>(
          d_wm_.p, m_off_[r][l], h.width[l + 1], h.full_cols[l], d_w_.p, d.w_off[l], d.pitch[l], l,
          h.n_v, h.pos_pad, p_.n_sin_waves, p_.duplicate_v, p_.duplicate_h, p_.duplicate_c);
    });
    transpose_weights();
  }

  // ---------------------------------------------------------------- I/O
  void upload_doubles(const double* host, size_t n) {
    CLS_REQUIRE(n <= d_stage_.n, "staging buffer too small");
    CLS_CUDA(cudaMemcpyAsync(d_stage_.p, host, sizeof(double) * n, cudaMemcpyHostToDevice, stream));
  }

  template <typename T>
  static int blocks_for(T n) { return (int)std::max<long long>(1, std::min<long long>(4096, ((long long)n + 255) / 256)); }

  // user-order [V][3] <-> internal-order [V][3]
  void to_internal(const double* in, std::vector<double>& out) const {
    out.resize((size_t)V_ * 3);
    for (int ie = 0; ie < E_; ++ie) {
      const int ue = perm_[ie];
      std::memcpy(&out[(size_t)ed_host_[ie].v_off * 3], in + (size_t)user_voff_[ue] * 3,
                  sizeof(double) * 3 * rd_host_[ed_host_[ie].robot].n_v);
    }
  }
  void to_user(const std::vector<double>& in, double* out) const {
    for (int ie = 0; ie < E_; ++ie) {
      const int ue = perm_[ie];
      std::memcpy(out + (size_t)user_voff_[ue] * 3, &in[(size_t)ed_host_[ie].v_off * 3],
                  sizeof(double) * 3 * rd_host_[ed_host_[ie].robot].n_v);
    }
  }

  void set_vstate(const double* host, V4<R>* dst) {
    const double* src = host;
    std::vector<double> tmp;
    if (!identity_perm_) { to_internal(host, tmp); src = tmp.data(); }
    upload_doubles(src, (size_t)V_ * 3);
    ms_xyz_to_v4_kernel<R><<<blocks_for(V_), 256, 0, stream>>>(d_stage_.p, dst, V_);
    CLS_CUDA(cudaGetLastError());
    if (!identity_perm_) CLS_CUDA(cudaStreamSynchronize(stream));  // tmp lifetime
  }

  void get_vstate(const V4<R>* srcd, double* host) {
    ms_v4_to_xyz_kernel<R><<<blocks_for(V_), 256, 0, stream>>>(srcd, d_stage_.p, V_);
    CLS_CUDA(cudaGetLastError());
    if (identity_perm_) {
      CLS_CUDA(cudaMemcpyAsync(host, d_stage_.p, sizeof(double) * V_ * 3, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    } else {
      std::vector<double> tmp((size_t)V_ * 3);
      CLS_CUDA(cudaMemcpyAsync(tmp.data(), d_stage_.p, sizeof(double) * V_ * 3, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
      to_user(tmp, host);
    }
  }

  void set_state(const double* x0, const double* v0) override {
    CLS_REQUIRE(x0 != nullptr, "x0 is required");
    set_vstate(x0, d_ckx_.p);
    CLS_CUDA(cudaMemcpyAsync(d_init_.p, d_ckx_.p, sizeof(V4<R>) * V_, cudaMemcpyDeviceToDevice, stream));
    if (v0) set_vstate(v0, d_ckv_.p);
    else CLS_CUDA(cudaMemsetAsync(d_ckv_.p, 0, sizeof(V4<R>) * V_, stream));
    fwd_done_ = bwd_done_ = false;
  }

  // [T][user env] -> [T][internal env]
  void permute_te(const double* in, int width, std::vector<double>& out) const {
    out.resize((size_t)T_ * E_ * width);
    for (int t = 0; t < T_; ++t)
      for (int ie = 0; ie < E_; ++ie)
        std::memcpy(&out[((size_t)t * E_ + ie) * width], in + ((size_t)t * E_ + perm_[ie]) * width,
                    sizeof(double) * width);
  }

  void set_targets(const double* tv, const double* th, const double* tc) override {
    std::vector<double> tmp;
    if (tv) {
      const double* src = tv;
      if (!identity_perm_) { permute_te(tv, 3, tmp); src = tmp.data(); }
      upload_doubles(src, (size_t)T_ * E_ * 3);
      ms_xyz_to_v4_kernel<R><<<blocks_for(T_ * E_), 256, 0, stream>>>(d_stage_.p, d_tv_.p, (long long)T_ * E_);
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    const double* arrs[2] = {th, tc};
    R* dsts[2] = {d_th_.p, d_tc_.p};
    for (int q = 0; q < 2; ++q) {
      if (!arrs[q]) {
        CLS_CUDA(cudaMemsetAsync(dsts[q], 0, sizeof(R) * (size_t)T_ * E_, stream));
        continue;
      }
      const double* src = arrs[q];
      if (!identity_perm_) { permute_te(arrs[q], 1, tmp); src = tmp.data(); }
      upload_doubles(src, (size_t)T_ * E_);
      ms_convert_kernel<R><<<blocks_for(T_ * E_), 256, 0, stream>>>(d_stage_.p, dsts[q], (long long)T_ * E_);
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    CLS_CUDA(cudaGetLastError());
  }

  void check_layer(int r, int l) const {
    CLS_REQUIRE(r >= 0 && r < (int)hr_.size(), "robot index out of range");
    CLS_REQUIRE(l >= 0 && l < L_, "layer index out of range");
  }

  void set_weights(int r, int l, const double* W, const double* b) override {
    check_layer(r, l);
    const HostRobot& h = hr_[r];
    const long long n = (long long)h.width[l + 1] * h.full_cols[l];
    if (W) {
      upload_doubles(W, n);
      ms_convert_kernel<R><<<blocks_for(n), 256, 0, stream>>>(d_stage_.p, d_wm_.p + m_off_[r][l], n);
      pack_layer(r, l);
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    if (b) {
      upload_doubles(b, h.width[l + 1]);
      ms_convert_kernel<R><<<1, 256, 0, stream>>>(d_stage_.p, d_bias_.p + rd_host_[r].b_off[l], h.width[l + 1]);
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    CLS_CUDA(cudaGetLastError());
  }

  void get_weights(int r, int l, double* W, double* b) override {
    check_layer(r, l);
    const HostRobot& h = hr_[r];
    const long long n = (long long)h.width[l + 1] * h.full_cols[l];
    if (W) {
      ms_to_double_kernel<R><<<blocks_for(n), 256, 0, stream>>>(d_wm_.p + m_off_[r][l], d_stage_.p, n);
      CLS_CUDA(cudaMemcpyAsync(W, d_stage_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    if (b) {
      ms_to_double_kernel<R><<<1, 256, 0, stream>>>(d_bias_.p + rd_host_[r].b_off[l], d_stage_.p, h.width[l + 1]);
      CLS_CUDA(cudaMemcpyAsync(b, d_stage_.p, sizeof(double) * h.width[l + 1], cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
  }

  void get_grads(int r, int l, double* gW, double* gb) override {
    check_layer(r, l);
    CLS_REQUIRE(bwd_done_, "gradients requested before cls_backward");
    const HostRobot& h = hr_[r];
    const RobotDesc& d = rd_host_[r];
    const long long n = (long long)h.width[l + 1] * h.full_cols[l];
    if (gW) {
      ms_unpack_grad_kernel<R><<<blocks_for(n), 256, 0, stream>>>(
          d_gw_.p, d.w_off[l], d.pitch[l], h.width[l + 1], h.full_cols[l], l, h.n_v, h.pos_pad,
          p_.n_sin_waves, p_.duplicate_v, p_.duplicate_h, p_.duplicate_c, d_stage_.p);
      CLS_CUDA(cudaMemcpyAsync(gW, d_stage_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    if (gb) {
      ms_to_double_kernel<R><<<1, 256, 0, stream>>>(d_gb_.p + d.b_off[l], d_stage_.p, h.width[l + 1]);
      CLS_CUDA(cudaMemcpyAsync(gb, d_stage_.p, sizeof(double) * h.width[l + 1], cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
  }

  void observables(double* c, double* h, double* u, double* rot) override {
    const long long n = (long long)T_ * E_;
    auto fetch_scalar = [&](const R* src, double* dst) {
      if (!dst) return;
      ms_to_double_kernel<R><<<blocks_for(n), 256, 0, stream>>>(src, d_stage_.p, n);
      std::vector<double> tmp(n);
      CLS_CUDA(cudaMemcpyAsync(tmp.data(), d_stage_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
      for (int t = 0; t < T_; ++t)
        for (int ie = 0; ie < E_; ++ie) dst[(size_t)t * E_ + perm_[ie]] = tmp[(size_t)t * E_ + ie];
    };
    if (c) {
      ms_v4_to_xyz_kernel<R><<<blocks_for(n), 256, 0, stream>>>(d_obsc_.p, d_stage_.p, n);
      std::vector<double> tmp(n * 3);
      CLS_CUDA(cudaMemcpyAsync(tmp.data(), d_stage_.p, sizeof(double) * n * 3, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
      for (int t = 0; t < T_; ++t)
        for (int ie = 0; ie < E_; ++ie)
          std::memcpy(c + ((size_t)t * E_ + perm_[ie]) * 3, &tmp[((size_t)t * E_ + ie) * 3], sizeof(double) * 3);
    }
    fetch_scalar(d_obsh_.p, h);
    fetch_scalar(d_obsu_.p, u);
    fetch_scalar(d_obsr_.p, rot);
  }

  void grad_buffers(void** w, long long* nw, void** b, long long* nb, int* elem) override {
    *w = d_gw_.p;
    *nw = (long long)d_gw_.n;
    *b = d_gb_.p;
    *nb = (long long)d_gb_.n;
    *elem = (int)sizeof(R);
  }

  // One substep of every env with outputs from the caller (external policy),
  // or (outputs == null, t == 0) the observation of the state set by
  // set_state.  outputs [E][omax] and obs [E][imax] in user env order, aux
  // [E][4] (centre, height of t).
  void env_step(int t, const double* outputs, double* obs, double* aux) override {
    CLS_REQUIRE(!capturing_, "not during graph capture");
    CLS_REQUIRE(t >= 0 && t < T_, "t out of range");
    CLS_REQUIRE(outputs != nullptr || t == 0, "without outputs only t = 0 (the initial observation)");
    CLS_REQUIRE(outputs == nullptr || t >= 1, "a step produces t >= 1");
    int omax = 1, imax = 1;
    for (const HostRobot& h : hr_) {
      omax = std::max(omax, h.width[h.n_layers]);
      imax = std::max(imax, h.full_cols[0]);
    }
    if (!d_livex_.p) { d_livex_.alloc(V_); d_livev_.alloc(V_); }
    if (d_envout_.n < (size_t)E_ * omax) d_envout_.alloc((size_t)E_ * omax);
    if (d_envobs_.n < (size_t)E_ * imax) d_envobs_.alloc((size_t)E_ * imax);
    if (d_envaux_.n < (size_t)E_ * 4) d_envaux_.alloc((size_t)E_ * 4);
    if (outputs) {
      std::vector<R> o((size_t)E_ * omax, R(0));
      for (int ie = 0; ie < E_; ++ie) {
        const int ue = perm_[ie], no = hr_[ed_host_[ie].robot].width[hr_[ed_host_[ie].robot].n_layers];
        for (int q = 0; q < no; ++q) o[(size_t)ie * omax + q] = (R)outputs[(size_t)ue * omax + q];
      }
      CLS_CUDA(cudaMemcpyAsync(d_envout_.p, o.data(), sizeof(R) * o.size(), cudaMemcpyHostToDevice, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    MsArgs<R> a = args(T_);
    a.w_smem = 0;
    a.b_smem = 0;
    a.live_x = d_livex_.p;
    a.live_v = d_livev_.p;
    const size_t smem = fwd_smem_bytes<R>(nmax_, smem_dmax_, smem_p0max_, imp_cap_);
    CLS_CUDA(EnvLaunch<R>::step(a, smem, stream, t, outputs ? 0 : 1, outputs ? d_envout_.p : nullptr, omax,
                                d_envobs_.p, imax, d_envaux_.p));
    std::vector<R> ob((size_t)E_ * imax), ax((size_t)E_ * 4);
    CLS_CUDA(cudaMemcpyAsync(ob.data(), d_envobs_.p, sizeof(R) * ob.size(), cudaMemcpyDeviceToHost, stream));
    CLS_CUDA(cudaMemcpyAsync(ax.data(), d_envaux_.p, sizeof(R) * ax.size(), cudaMemcpyDeviceToHost, stream));
    CLS_CUDA(cudaStreamSynchronize(stream));
    for (int ie = 0; ie < E_; ++ie) {
      const int ue = perm_[ie];
      if (obs)
        for (int q = 0; q < imax; ++q) obs[(size_t)ue * imax + q] = (double)ob[(size_t)ie * imax + q];
      if (aux)
        for (int q = 0; q < 4; ++q) aux[(size_t)ue * 4 + q] = (double)ax[(size_t)ie * 4 + q];
    }
    fwd_done_ = bwd_done_ = false;
  }

  // targets of one env for t in [t_from, T), other times and envs untouched
  void env_set_targets(int ue, int t_from, const double* tv, const double* th, const double* tc) override {
    const int ie = ienv(ue);
    CLS_REQUIRE(t_from >= 0 && t_from < T_, "t_from out of range");
    const int n = T_ - t_from;
    if (tv) {
      std::vector<V4<R>> v(n);
      for (int t = 0; t < n; ++t) {
        v[t].x = (R)tv[3 * t]; v[t].y = (R)tv[3 * t + 1]; v[t].z = (R)tv[3 * t + 2]; v[t].w = 0;
      }
      CLS_CUDA(cudaMemcpy2DAsync(d_tv_.p + (size_t)t_from * E_ + ie, sizeof(V4<R>) * E_, v.data(), sizeof(V4<R>),
                                 sizeof(V4<R>), n, cudaMemcpyHostToDevice, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
    const double* src[2] = {th, tc};
    R* dst[2] = {d_th_.p, d_tc_.p};
    for (int q = 0; q < 2; ++q) {
      if (!src[q]) continue;
      std::vector<R> v(n);
      for (int t = 0; t < n; ++t) v[t] = (R)src[q][t];
      CLS_CUDA(cudaMemcpy2DAsync(dst[q] + (size_t)t_from * E_ + ie, sizeof(R) * E_, v.data(), sizeof(R), sizeof(R),
                                 n, cudaMemcpyHostToDevice, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
    }
  }

  void debug_gemm_starve(int starve, unsigned wait_limit) override {
    CLS_REQUIRE(!capturing_, "not during graph capture");
    gemm_starve_ = starve ? 1 : 0;
    gemm_wait_limit_ = wait_limit;
  }

  void set_loss_envs(int r, int n) override {
    CLS_REQUIRE(r >= 0 && r < (int)rd_host_.size(), "robot index out of range");
    CLS_REQUIRE(n >= rd_host_[r].n_env && n > 0,
                "the loss env count must be at least the handle's env count of the type");
    CLS_REQUIRE(!capturing_, "the loss normalisation cannot change during graph capture");
    if (rd_host_[r].loss_envs == n) return;
    rd_host_[r].loss_envs = n;
    CLS_CUDA(cudaMemcpyAsync(d_robots_.p + r, &rd_host_[r], sizeof(RobotDesc), cudaMemcpyHostToDevice,
                             stream));
    CLS_CUDA(cudaStreamSynchronize(stream));
    fwd_done_ = false;
    bwd_done_ = false;
  }

  void set_loss_mask(int mask) override {
    CLS_REQUIRE((mask & ~(LOSS_VELOCITY | LOSS_HEIGHT | LOSS_POSE | LOSS_ACTUATION | LOSS_ROTATION |
                          LOSS_CRAWL)) == 0,
                "unknown loss bits");
    CLS_REQUIRE(!(mask & (LOSS_ROTATION | LOSS_POSE)) || d_xfull_.p != nullptr,
                "rotation and pose losses need the trajectory: create the handle with one of them or "
                "with keep_trajectory");
    CLS_REQUIRE(!(mask & LOSS_ACTUATION) || d_actfull_.p != nullptr,
                "the actuation loss needs its record: create the handle with it");
    CLS_REQUIRE(!capturing_, "the loss set cannot change during graph capture");
    if (mask == p_.loss_mask) return;
    p_.loss_mask = mask;
    fwd_done_ = false;
    bwd_done_ = false;
  }

  void targets(double* tv, double* th, double* tc) override {
    const long long n = (long long)T_ * E_;
    auto fetch_scalar = [&](const R* src, double* dst) {
      if (!dst) return;
      ms_to_double_kernel<R><<<blocks_for(n), 256, 0, stream>>>(src, d_stage_.p, n);
      std::vector<double> tmp(n);
      CLS_CUDA(cudaMemcpyAsync(tmp.data(), d_stage_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
      for (int t = 0; t < T_; ++t)
        for (int ie = 0; ie < E_; ++ie) dst[(size_t)t * E_ + perm_[ie]] = tmp[(size_t)t * E_ + ie];
    };
    if (tv) {
      ms_v4_to_xyz_kernel<R><<<blocks_for(n), 256, 0, stream>>>(d_tv_.p, d_stage_.p, n);
      std::vector<double> tmp(n * 3);
      CLS_CUDA(cudaMemcpyAsync(tmp.data(), d_stage_.p, sizeof(double) * n * 3, cudaMemcpyDeviceToHost, stream));
      CLS_CUDA(cudaStreamSynchronize(stream));
      for (int t = 0; t < T_; ++t)
        for (int ie = 0; ie < E_; ++ie)
          std::memcpy(tv + ((size_t)t * E_ + perm_[ie]) * 3, &tmp[((size_t)t * E_ + ie) * 3], sizeof(double) * 3);
    }
    fetch_scalar(d_th_.p, th);
    fetch_scalar(d_tc_.p, tc);
  }

  void trajectory(double* x) override {
    CLS_REQUIRE(d_xfull_.p != nullptr, "trajectory is only kept with a rotation or pose loss or keep_trajectory");
    for (int t = 0; t < T_; ++t) get_vstate(d_xfull_.p + (size_t)t * V_, x + (size_t)t * V_ * 3);
  }

  void final_state(double* x, double* v) override {
    if (x) get_vstate(d_finx_.p, x);
    if (v) get_vstate(d_finv_.p, v);
  }

  // ------------------------------------------------------------- serving
  // A served batch advances envs that sit at different times of their own
  // episodes: every launch takes a window {t_begin, t_end, source checkpoint,
  // first reverse segment} per env (user order; t_begin >= t_end: idle) and
  // per-env episode steps.  Envs keep their state, targets, observables and
  // checkpoints in their own regions, so admitting an env (serve_reset_env)
  // touches no other env.
  int ienv(int ue) const {
    CLS_REQUIRE(ue >= 0 && ue < E_, "env index out of range");
    return inv_perm_[ue];
  }

  void serve_reset_env(int ue, const double* x0, const double* v0, const double* tv, const double* th,
                       const double* tc) override {
    const int ie = ienv(ue);
    const EnvDesc& ed = ed_host_[ie];
    const int N = rd_host_[ed.robot].n_v;
    CLS_REQUIRE(x0 != nullptr, "x0 is required");
    std::vector<V4<R>> xs(N), vs(N);
    for (int i = 0; i < N; ++i) {
      xs[i].x = (R)x0[3 * i]; xs[i].y = (R)x0[3 * i + 1]; xs[i].z = (R)x0[3 * i + 2]; xs[i].w = 0;
      vs[i].x = v0 ? (R)v0[3 * i] : R(0); vs[i].y = v0 ? (R)v0[3 * i + 1] : R(0);
      vs[i].z = v0 ? (R)v0[3 * i + 2] : R(0); vs[i].w = 0;
    }
    CLS_CUDA(cudaMemcpyAsync(d_ckx_.p + ed.v_off, xs.data(), sizeof(V4<R>) * N, cudaMemcpyHostToDevice, stream));
    CLS_CUDA(cudaMemcpyAsync(d_init_.p + ed.v_off, xs.data(), sizeof(V4<R>) * N, cudaMemcpyHostToDevice, stream));
    CLS_CUDA(cudaMemcpyAsync(d_ckv_.p + ed.v_off, vs.data(), sizeof(V4<R>) * N, cudaMemcpyHostToDevice, stream));
    // targets: one column of the [T][E] arrays
    std::vector<V4<R>> tvv(T_);
    std::vector<R> thv(T_), tcv(T_);
    for (int t = 0; t < T_; ++t) {
      tvv[t].x = tv ? (R)tv[3 * t] : R(0); tvv[t].y = tv ? (R)tv[3 * t + 1] : R(0);
      tvv[t].z = tv ? (R)tv[3 * t + 2] : R(0); tvv[t].w = 0;
      thv[t] = th ? (R)th[t] : R(0);
      tcv[t] = tc ? (R)tc[t] : R(0);
    }
    CLS_CUDA(cudaMemcpy2DAsync(d_tv_.p + ie, sizeof(V4<R>) * E_, tvv.data(), sizeof(V4<R>), sizeof(V4<R>), T_,
                               cudaMemcpyHostToDevice, stream));
    CLS_CUDA(cudaMemcpy2DAsync(d_th_.p + ie, sizeof(R) * E_, thv.data(), sizeof(R), sizeof(R), T_,
                               cudaMemcpyHostToDevice, stream));
    CLS_CUDA(cudaMemcpy2DAsync(d_tc_.p + ie, sizeof(R) * E_, tcv.data(), sizeof(R), sizeof(R), T_,
                               cudaMemcpyHostToDevice, stream));
    // observables and trajectories of the env start at zero, as after the
    // whole-batch clears of cls_forward
    CLS_CUDA(cudaMemset2DAsync(d_obsc_.p + ie, sizeof(V4<R>) * E_, 0, sizeof(V4<R>), T_, stream));
    CLS_CUDA(cudaMemset2DAsync(d_obsh_.p + ie, sizeof(R) * E_, 0, sizeof(R), T_, stream));
    CLS_CUDA(cudaMemset2DAsync(d_obsu_.p + ie, sizeof(R) * E_, 0, sizeof(R), T_, stream));
    CLS_CUDA(cudaMemset2DAsync(d_obsr_.p + ie, sizeof(R) * E_, 0, sizeof(R), T_, stream));
    if (d_xfull_.p)
      CLS_CUDA(cudaMemset2DAsync(d_xfull_.p + ed.v_off, sizeof(V4<R>) * V_, 0, sizeof(V4<R>) * N, T_, stream));
    if (d_actfull_.p) {
      const int zt = z_total_[L_ - 1], no = rd_host_[ed.robot].n_out;
      CLS_CUDA(cudaMemset2DAsync(d_actfull_.p + ed.z_off[L_ - 1], sizeof(R) * zt, 0, sizeof(R) * no, T_, stream));
    }
    CLS_CUDA(cudaStreamSynchronize(stream));  // host staging vectors go out of scope
  }

  // windows and steps (user order) -> internal tables in one staging slot
  // (int4 windows [E], int steps [E], int order [E]); returns the active
  // count; the slot's device address is left in serve_stage_.
  int serve_prepare(const int* win, const int* steps, bool reverse) {
    CLS_REQUIRE(win != nullptr && steps != nullptr, "windows and steps are required");
    std::vector<int4>& w = serve_w_tmp_;
    std::vector<int>& st = serve_st_tmp_;
    std::vector<int>& order = serve_order_h_;
    w.assign(E_, make_int4(0, 0, 0, 0));
    st.assign(E_, 0);
    order.clear();
    for (int ie = 0; ie < E_; ++ie) {
      const int ue = perm_[ie];
      w[ie] = make_int4(win[4 * ue], win[4 * ue + 1], win[4 * ue + 2], win[4 * ue + 3]);
      st[ie] = steps[ue];
      if (w[ie].x < w[ie].y) {
        CLS_REQUIRE(st[ie] >= 2 && st[ie] <= T_, "episode steps out of range");
        CLS_REQUIRE(w[ie].x >= 0 && w[ie].y <= st[ie] - 1, "a window lies in [0, steps - 1)");
        CLS_REQUIRE(!reverse || w[ie].y - w[ie].x <= K_, "a reverse window spans one checkpoint segment");
        CLS_REQUIRE(w[ie].z >= 0 && w[ie].z < (int)n_ckpt_ && w[ie].x == w[ie].z * K_,
                    "a window starts at its source checkpoint (t_begin = checkpoint * checkpoint_every)");
      }
    }
    for (int ie : order_host_)
      if (w[ie].x < w[ie].y) order.push_back(ie);
    if (!stage_.host) CLS_CUDA(stage_.init(stage_bytes()));
    unsigned char *h, *d;
    int slot;
    CLS_CUDA(stage_.acquire(&h, &d, &slot));
    std::memcpy(h, w.data(), sizeof(int4) * E_);
    std::memcpy(h + sizeof(int4) * E_, st.data(), sizeof(int) * E_);
    std::memcpy(h + (sizeof(int4) + sizeof(int)) * E_, order.data(), sizeof(int) * order.size());
    CLS_CUDA(stage_.upload(slot, (sizeof(int4) + 2 * sizeof(int)) * E_, stream));
    serve_stage_ = d;
    serve_win_h_ = w;
    return (int)order.size();
  }

  size_t stage_bytes() const {
    return std::max((sizeof(int4) + 2 * sizeof(int)) * (size_t)E_,
                    sizeof(GemmTile) * std::max<size_t>(1, tiles_host_.size()));
  }

  MsArgs<R> serve_args(int n) {
    MsArgs<R> a = args(T_);
    a.win = reinterpret_cast<const int4*>(serve_stage_);
    a.env_steps = reinterpret_cast<const int*>(serve_stage_ + sizeof(int4) * E_);
    a.order = reinterpret_cast<const int*>(serve_stage_ + (sizeof(int4) + sizeof(int)) * E_);
    a.n_items = n;
    return a;
  }

  void serve_forward(const int* win, const int* steps) override {
    const int n = serve_prepare(win, steps, false);
    if (n == 0) return;
    CLS_CUDA(cudaMemsetAsync(d_squeue_.p, 0, sizeof(int) * 2, stream));
    MsArgs<R> a = serve_args(n);
    a.queue = d_squeue_.p;
    timed(PK_FWD, [&] {
      fwd_fn()<<<grid_for(n), threads_, fwd_smem_, stream>>>(a, 0, 0, FWD_CKPT | FWD_OBS | FWD_CKEND, 0);
    });
    CLS_CUDA(cudaGetLastError());
  }

  void serve_backward(const int* win, const int* steps) override {
    const int n = serve_prepare(win, steps, true);
    if (n == 0) return;
    // a robot's weight gradients restart with its env's first reverse segment
    std::vector<int> active_robot(rd_host_.size(), 0);
    for (int ie : serve_order_h_) {
      const int r = ed_host_[ie].robot;
      CLS_REQUIRE(rd_host_[r].n_env == 1, "served envs need a robot (controller) of their own");
      active_robot[r] = 1;
      if (serve_win_h_[ie].w) {
        const RobotDesc& d = rd_host_[r];
        const long long w0 = d.w_off[0];
        const long long w1 = d.w_off[L_ - 1] + (long long)d.pitch[L_ - 1] * d.width[L_];
        const int b0 = d.b_off[0], b1 = d.b_off[L_ - 1] + d.width[L_];
        CLS_CUDA(cudaMemsetAsync(d_gw_.p + w0, 0, sizeof(R) * (w1 - w0), stream));
        CLS_CUDA(cudaMemsetAsync(d_gb_.p + b0, 0, sizeof(R) * (b1 - b0), stream));
      }
    }
    std::vector<GemmTile> tiles;
    for (const GemmTile& t : tiles_host_)
      if (active_robot[t.robot]) tiles.push_back(t);
    CLS_CUDA(cudaMemsetAsync(d_squeue_.p, 0, sizeof(int) * 2, stream));
    MsArgs<R> a = serve_args(n);
    a.queue = d_squeue_.p;
    timed(PK_RECOMP, [&] { fwd_fn()<<<grid_for(n), threads_, fwd_smem_, stream>>>(a, 0, 0, FWD_RECORD, 0); });
    a.queue = d_squeue_.p + 1;
    timed(PK_REV, [&] { rev_fn()<<<grid_for(n), threads_, rev_smem_, stream>>>(a, 0, 0, 0); });
    if (!tiles.empty()) {
      unsigned char *h, *d;
      int slot;
      CLS_CUDA(stage_.acquire(&h, &d, &slot));
      std::memcpy(h, tiles.data(), sizeof(GemmTile) * tiles.size());
      CLS_CUDA(stage_.upload(slot, sizeof(GemmTile) * tiles.size(), stream));
      const GemmTile* dt = reinterpret_cast<const GemmTile*>(d);
      timed(PK_WGRAD, [&] {
        ms_wgrad_kernel<R><<<(int)tiles.size(), 256, 0, stream>>>(a, dt, 0, d_gw_.p, d_gb_.p);
      });
    }
    CLS_CUDA(cudaGetLastError());
    bwd_done_ = true;  // served robots' gradients are readable (cls_get_grads)
  }

  void serve_loss(const int* steps, double* env) override {
    CLS_REQUIRE(steps != nullptr, "steps are required");
    std::vector<int> st(E_), list;
    for (int ie = 0; ie < E_; ++ie) {
      st[ie] = steps[perm_[ie]];
      if (st[ie] <= 0) continue;  // not requested
      CLS_REQUIRE(st[ie] >= 2 && st[ie] <= T_, "episode steps out of range");
      list.push_back(ie);
    }
    CLS_CUDA(cudaMemsetAsync(d_lossenv_.p, 0, sizeof(double) * E_ * 8, stream));
    if (!list.empty()) {
      CLS_CUDA(cudaMemcpyAsync(d_env_steps_.p, st.data(), sizeof(int) * E_, cudaMemcpyHostToDevice, stream));
      CLS_CUDA(cudaMemcpyAsync(d_sorder_.p, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice,
                               stream));
      MsArgs<R> a = args(T_);
      a.env_steps = d_env_steps_.p;
      timed(PK_LOSS, [&] {
        ms_loss_kernel<R><<<(int)list.size(), 256, 0, stream>>>(a, d_lossenv_.p, d_sorder_.p);
      });
      CLS_CUDA(cudaGetLastError());
    }
    std::vector<double> raw((size_t)E_ * 8);
    CLS_CUDA(cudaMemcpyAsync(raw.data(), d_lossenv_.p, sizeof(double) * raw.size(), cudaMemcpyDeviceToHost, stream));
    CLS_CUDA(cudaStreamSynchronize(stream));
    loss_from_raw(raw, nullptr, env);
  }

  void serve_env_state(int ue, double* x, double* v) override {
    const int ie = ienv(ue);
    const EnvDesc& ed = ed_host_[ie];
    const int N = rd_host_[ed.robot].n_v;
    std::vector<V4<R>> xs(N), vs(N);
    CLS_CUDA(cudaMemcpyAsync(xs.data(), d_finx_.p + ed.v_off, sizeof(V4<R>) * N, cudaMemcpyDeviceToHost, stream));
    CLS_CUDA(cudaMemcpyAsync(vs.data(), d_finv_.p + ed.v_off, sizeof(V4<R>) * N, cudaMemcpyDeviceToHost, stream));
    CLS_CUDA(cudaStreamSynchronize(stream));
    for (int i = 0; i < N; ++i) {
      if (x) { x[3 * i] = (double)xs[i].x; x[3 * i + 1] = (double)xs[i].y; x[3 * i + 2] = (double)xs[i].z; }
      if (v) { v[3 * i] = (double)vs[i].x; v[3 * i + 1] = (double)vs[i].y; v[3 * i + 2] = (double)vs[i].z; }
    }
  }

  // robot class of every robot entry: the first entry with the same
  // geometry, spring table, output map and layer widths (computed once)
  int env_class(int ue) const override {
    if (robot_class_.empty()) {
      const int nr = (int)hr_.size();
      robot_class_.assign(nr, 0);
      for (int r = 0; r < nr; ++r) {
        robot_class_[r] = r;
        for (int q = 0; q < r; ++q)
          if (robot_class_[q] == q && same_robot(hr_[q], hr_[r])) { robot_class_[r] = q; break; }
      }
    }
    return robot_class_[ed_host_[ienv(ue)].robot];
  }
  static bool same_robot(const HostRobot& a, const HostRobot& b) {
    if (a.n_v != b.n_v || a.n_s != b.n_s || a.n_out != b.n_out || a.robot_id != b.robot_id ||
        a.n_layers != b.n_layers)
      return false;
    for (int l = 0; l <= a.n_layers; ++l)
      if (a.width[l] != b.width[l]) return false;
    return a.objects == b.objects && a.sa == b.sa && a.sb == b.sb && a.out == b.out && a.len == b.len &&
           a.stiff == b.stiff && a.coef == b.coef;
  }
  int env_vertices(int ue) const override { return hr_[ed_host_[ienv(ue)].robot].n_v; }
  bool env_own_robot(int ue) const override { return rd_host_[ed_host_[ienv(ue)].robot].n_env == 1; }
  const double* env_objects(int ue) const override { return hr_[ed_host_[ienv(ue)].robot].objects.data(); }
  // HBM bytes a request keeps resident while it is served (the terms of
  // serving.footprint_bytes over this handle's own layer widths, the input
  // layer in its compact form): state and checkpoints, trajectory and
  // observables, targets, controller weights (x3 with gradient and
  // optimiser-sized buffers) and, for gradient queries, the per-segment
  // records of its reverse pass
  long long env_footprint(int ue, int steps, bool grad) const override {
    const HostRobot& h = hr_[ed_host_[ienv(ue)].robot];
    const long long n = h.n_v, K = K_;
    long long params = 0, widths_after = 0;
    for (int l = 0; l < h.n_layers; ++l) {
      params += (long long)h.width[l + 1] * h.width[l] + h.width[l + 1];
      widths_after += h.width[l + 1];
    }
    const long long ckpt = 2 * 16 * n * (steps / K + 2);
    const long long traj = 16 * n * steps + 32LL * steps + 24LL * steps;
    const long long w = params * (long long)sizeof(R) * (grad ? 3 : 1);
    const long long rec = grad ? K * (48 * n + 8 * widths_after + 4LL * h.width[0]) : 0;
    return ckpt + traj + w + rec;
  }
  int checkpoint_every() const override { return K_; }

  void state_grads(double* gx, double* gv) override {
    CLS_REQUIRE(bwd_done_, "state gradients requested before cls_backward");
    if (gx) get_vstate(d_adjx_.p, gx);
    if (gv) get_vstate(d_adjv_.p, gv);
  }

  int synchronize() override {
    CLS_CUDA(cudaStreamSynchronize(stream));
    int st = 0;
    CLS_CUDA(cudaMemcpy(&st, d_status_.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (st) {
      CLS_CUDA(cudaMemset(d_status_.p, 0, sizeof(int)));
      // a timeout first: the results after it are invalid anyway
      if (st & ERR_TIMEOUT) {
        err = (st & ERR_NONFINITE)
                  ? "a tensor-core GEMM tile's bounded wait for its operands or MMAs ran out (the tile "
                    "freed its tensor memory and skipped its epilogue); non-finite state was seen too"
                  : "a tensor-core GEMM tile's bounded wait for its operands or MMAs ran out; the tile "
                    "freed its tensor memory and skipped its epilogue";
        return CLS_ERR_TIMEOUT;
      }
      if (st & ERR_NONFINITE) {
        err = "non-finite state detected";
        return CLS_ERR_NONFINITE;
      }
    }
    return CLS_OK;
  }

  void graph_capture(int steps, bool with_adam) override {
    CLS_REQUIRE(stream != nullptr, "graph capture needs a non-default stream (cls_set_stream)");
    if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
    CLS_REQUIRE(!prof_.on, "disable profiling before graph capture");
    CLS_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing_ = true;
    try {
      forward(steps, false, false);
      loss_device();
      backward(false);
      if (with_adam) adam_device(-1, true, d_tns_.p);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      capturing_ = false;
      throw;
    }
    capturing_ = false;
    CLS_CUDA(cudaStreamEndCapture(stream, &graph_));
    CLS_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0));
    graph_adam_ = with_adam;
  }

  void graph_launch(int iter) override {
    CLS_REQUIRE(graph_exec_ != nullptr, "no captured graph (cls_graph_capture)");
    if (graph_adam_) {
      iter_host_ = iter;
      CLS_CUDA(cudaMemcpyAsync(d_iter_.p, &iter_host_, sizeof(int), cudaMemcpyHostToDevice, stream));
    }
    CLS_CUDA(cudaGraphLaunch(graph_exec_, stream));
  }

  void sizes(int* ne, int* nv, int* T) const override {
    if (ne) *ne = E_;
    if (nv) *nv = V_;
    if (T) *T = T_;
  }
  void layer_shape(int r, int l, int* rows, int* cols) const override {
    check_layer(r, l);
    if (rows) *rows = hr_[r].width[l + 1];
    if (cols) *cols = hr_[r].full_cols[l];
  }


 private:
  std::vector<HostRobot> hr_;
  cls_sim_params p_;
  int E_ = 0, T_ = 0, K_ = 1, L_ = 1, V_ = 0, in_total_ = 0, nmax_ = 0;
  int z_total_[kMaxLayers] = {0};
  long long z_base_[kMaxLayers] = {0};
  long long rec_z_total_ = 0;
  mutable std::vector<int> robot_class_;  // env_class: first robot entry of each entry's class
  int smem_p0max_ = 0, smem_dmax_ = 0, smem_amax_ = 0, smem_omax_ = 0, threads_ = 256, n_sm_ = 148, n_ckpt_ = 0;
  int ctas_per_sm_ = 2, resident_ = 1;
  // controller span of the largest robot (elements) and whether the fused
  // kernels keep it in shared memory; forward shared memory without it
  long long wspan_max_ = 0, bspan_max_ = 0;
  bool wsh_on_ = false;
  size_t fwd_base_ = 0;
  size_t fwd_smem_ = 0, rev_smem_ = 0, n_queue_ = 0;
  std::vector<int> perm_, user_voff_, env_robot_, order_host_;
  bool identity_perm_ = true;
  std::vector<EnvDesc> ed_host_;
  std::vector<RobotDesc> rd_host_;
  std::vector<GemmTile> tiles_host_;
  std::vector<GemmTile> tiles_ep_;  // weight-gradient tiles over whole-episode records
  int rec_slots_ = 1;               // controller-record slots (K, or one per substep)
  bool episode_records() const { return rec_slots_ > K_ && !tiles_ep_.empty(); }
  // the first pass recorded the last segment (FWD_RECTAIL), in the
  // whole-episode layout when tail_episode_
  bool tail_recorded_ = false, tail_episode_ = false;
  std::vector<int> inv_perm_, serve_order_h_, serve_st_tmp_;
  std::vector<int4> serve_win_h_, serve_w_tmp_;
  DevBuf<int> d_env_steps_, d_sorder_, d_squeue_;
  StageRing stage_;
  unsigned char* serve_stage_ = nullptr;
  std::vector<OptSeg> opt_segs_, pack_segs_;
  long long opt_total_ = 0, pack_total_ = 0;
  double tns_host_ = 0;
  std::vector<std::vector<long long>> m_off_;
  bool keep_x_ = false, fwd_done_ = false, bwd_done_ = false, eval_ = false, per_env_ = false;
  bool graph_adam_ = false, capturing_ = false;
  unsigned gemm_wait_limit_ = 0;
  int gemm_starve_ = 0;
  Profiler prof_;
  int steps_ = 0, qslot_ = 0, iter_host_ = 0;
  double max_height_ = 0;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  DevBuf<RobotDesc> d_robots_;
  DevBuf<EnvDesc> d_envs_;
  DevBuf<int> d_order_, d_queue_, d_inc_ptr_, d_spring_out_, d_status_, d_iter_;
  DevBuf<int4> d_inc_i_, d_inc_p_, d_spr_ab_;
  DevBuf<V4<R>> d_spr_p_;
  size_t imp_cap_ = 0;
  int smax_ = 0;
  static constexpr size_t kImpSmemMax = 48 * 1024;
  DevBuf<V4<R>> d_inc_f_, d_ckx_, d_ckv_, d_finx_, d_finv_, d_recx_, d_recv_, d_recvinc_, d_obsc_, d_xfull_,
      d_tv_, d_init_, d_adjx_, d_adjv_;
  DevBuf<R> d_w_, d_gw_, d_bias_, d_gb_, d_bm_, d_bv_, d_wm_, d_wmm_, d_wmv_, d_sin_, d_recin_,
      d_recz_, d_recdz_, d_obsh_, d_obsu_, d_obsr_, d_actfull_, d_th_, d_tc_, d_adjh_;
  DevBuf<unsigned char> d_head_;
  DevBuf<unsigned long long> d_phase_;
  // batched controller path
  bool dense_ = false;
  int dense_threads_ = 128, n_ttiles_ = 0;
  size_t dfwd_smem_ = 0, drev_smem_ = 0;
  long long wt_total_ = 0;
  std::vector<TransSeg> tsegs_;
  std::vector<DenseJob> jobs_h_;
  int jf_off_[kMaxLayers] = {0}, jf_cnt_[kMaxLayers] = {0}, jb_off_[kMaxLayers] = {0}, jb_cnt_[kMaxLayers] = {0};
  DevBuf<DenseJob> d_jobs_;
  DevBuf<TransSeg> d_tsegs_;
  DevBuf<V4<R>> d_livex_, d_livev_;
  DevBuf<R> d_envout_, d_envobs_, d_envaux_;
  DevBuf<R> d_din_, d_wt_, d_split_;
  std::vector<DenseDesc> dd_host_;
  DevBuf<DenseDesc> d_dense_;
  // FP32 batched path: tensor-core weight-gradient products
  DevBuf<R> d_wsplit_;
  std::vector<WgTrans> wg_trans_;
  std::vector<WgCol> wg_cols_;
  std::vector<WgJob> wg_jobs_;
  DevBuf<WgTrans> d_wg_trans_;
  DevBuf<WgCol> d_wg_cols_;
  DevBuf<WgJob> d_wg_jobs_;
  int wg_grid_x_ = 0, wg_chunk_ = 1;
  // record slots per weight-gradient pass (bounds its operand buffers)
  static constexpr int kWgChunkSlots = 50;
  bool recorded_ = false;  // the first pass recorded the only segment
  std::vector<SplitSeg> ssegs_;
  DevBuf<SplitSeg> d_ssegs_;
  long long split_total_ = 0;

 public:
  void phase_read(unsigned long long* out) override {
    CLS_CUDA(cudaStreamSynchronize(stream));
    if (d_phase_.p) CLS_CUDA(cudaMemcpy(out, d_phase_.p, sizeof(unsigned long long) * 32, cudaMemcpyDeviceToHost));
    else std::memset(out, 0, sizeof(unsigned long long) * 32);
  }

 private:
  DevBuf<double> d_lossenv_, d_stage_, d_tns_;
  DevBuf<GemmTile> d_tiles_, d_tiles_ep_;
  DevBuf<OptSeg> d_opt_segs_, d_pack_segs_;
};

}  // namespace cls

namespace cls {

// The slot scheduler's operations over a served handle (cls_admit /
// cls_poll): the cls_serve_* primitives on the handle's stream.
class SimSlotOps final : public SlotOps {
 public:
  explicit SimSlotOps(SimBase& s) : s_(s) { s_.sizes(&E_, &nv_, &T_); }
  int n_slots() const override { return E_; }
  int max_steps() const override { return T_; }
  int checkpoint_every() const override { return s_.checkpoint_every(); }
  int slot_class(int slot) const override { return s_.env_class(slot); }
  int n_vertices(int slot) const override { return s_.env_vertices(slot); }
  bool own_controller(int slot) const override { return s_.env_own_robot(slot); }
  long long footprint(int slot, int steps, bool grad) const override {
    return s_.env_footprint(slot, steps, grad);
  }
  void reset(int slot, const double* x0, const double* tv, const double* th, const double* tc) override {
    s_.serve_reset_env(slot, x0 ? x0 : s_.env_objects(slot), nullptr, tv, th, tc);
  }
  void forward(const int* w, const int* st) override { s_.serve_forward(w, st); }
  void backward(const int* w, const int* st) override { s_.serve_backward(w, st); }
  void loss(const int* st, double* env) override { s_.serve_loss(st, env); }
  void final_x(int slot, double* x) override { s_.serve_env_state(slot, x, nullptr); }
  void wait() override {
    const int rc = s_.synchronize();
    if (rc != CLS_OK) throw Fail{rc, s_.err};
  }

 private:
  SimBase& s_;
  int E_ = 0, nv_ = 0, T_ = 0;
};

}  // namespace cls

// ===================================================================== C ABI
struct cls_sim {
  std::unique_ptr<cls::SimBase> impl;
  // continuous-batching scheduler, created by the first cls_admit /
  // cls_serve_tick (declared after impl: destroyed before it)
  std::unique_ptr<cls::SimSlotOps> slot_ops;
  std::unique_ptr<cls::SlotScheduler> sched;
  int tick_segments = 1;
};

namespace cls {
static SlotScheduler& scheduler(cls_sim* sim) {
  if (!sim->sched) {
    sim->slot_ops.reset(new SimSlotOps(*sim->impl));
    sim->sched.reset(new SlotScheduler(*sim->slot_ops, sim->tick_segments));
  }
  return *sim->sched;
}
}  // namespace cls

using cls::Fail;

template <typename F>
static int guarded(cls_sim* s, F&& f) {
  if (!s || !s->impl) return CLS_ERR_INVALID;
  try {
    f(*s->impl);
    return CLS_OK;
  } catch (const Fail& e) {
    s->impl->err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    s->impl->err = e.what();
    return CLS_ERR_INVALID;
  }
}

extern "C" {

void cls_default_params(cls_sim_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->max_steps = 1000;
  p->dt = 0.004;
  p->gravity = -1.8;
  p->ground_height = 0.1;
  p->drag_damping = 0.0;
  p->dashpot_damping = 0.1;
  p->friction = 0.4;
  p->stiffness_scale = 0.1;
  p->run_period = 100;
  p->turn_period = 500;
  p->jump_period = 500;
  p->spring_omega = 2 * M_PI / 0.004 / 100;
  p->n_sin_waves = 100;
  p->duplicate_v = 150;
  p->duplicate_h = 150;
  p->duplicate_c = 0;
  p->activation_hidden = CLS_ACT_SIN;
  p->activation_output = CLS_ACT_SIN;
  p->loss_mask = CLS_LOSS_VELOCITY | CLS_LOSS_ROTATION;
  p->precision = 32;
  p->checkpoint_every = 50;
  p->max_speed = 0.1;
  p->max_height = 0.1;
  p->adam_b1 = 0.9;
  p->adam_b2 = 0.9;
  p->learning_rate = 3e-4;
  p->threads_per_block = 0;
  p->keep_trajectory = 0;
}

int cls_create(const cls_robot_desc* robots, int32_t n_robots, const int32_t* env_robot,
               int32_t n_envs, const cls_sim_params* params, cls_sim** out) {
  using namespace cls;
  if (!out) return CLS_ERR_INVALID;
  *out = nullptr;
  try {
    CLS_REQUIRE(robots && n_robots > 0 && env_robot && n_envs > 0 && params, "null or empty argument");
    const cls_sim_params& p = *params;
    CLS_REQUIRE(p.precision == 32 || p.precision == 64, "precision must be 32 or 64");
    CLS_REQUIRE(p.max_steps >= 2, "max_steps must be >= 2");
    CLS_REQUIRE(p.run_period > 0 && p.turn_period > 0 && p.jump_period > 0, "periods must be > 0");
    CLS_REQUIRE(p.n_sin_waves >= 0 && p.duplicate_v >= 0 && p.duplicate_h >= 0 && p.duplicate_c >= 0,
                "negative input sizes");
    CLS_REQUIRE(p.activation_hidden == 0 || p.activation_hidden == 1, "bad hidden activation");
    CLS_REQUIRE(p.activation_output == 0 || p.activation_output == 1, "bad output activation");
    std::vector<HostRobot> hr(n_robots);
    int nl = -1;
    for (int r = 0; r < n_robots; ++r) {
      const cls_robot_desc& d = robots[r];
      HostRobot& h = hr[r];
      CLS_REQUIRE(d.n_vertices > 0 && d.objects && (d.n_springs == 0 || d.springs), "robot geometry missing");
      CLS_REQUIRE(d.n_hidden_layers >= 1 && d.n_hidden_layers <= CLS_MAX_HIDDEN, "1..4 hidden layers");
      if (nl < 0) nl = d.n_hidden_layers;
      CLS_REQUIRE(nl == d.n_hidden_layers, "all robots of a batch need the same MLP depth");
      h.n_v = d.n_vertices;
      h.n_s = d.n_springs;
      h.robot_id = d.robot_id;
      h.objects.assign(d.objects, d.objects + 3 * (size_t)d.n_vertices);
      h.n_out = d.n_outputs > 0 ? d.n_outputs : d.n_springs;
      CLS_REQUIRE(h.n_out > 0, "robot has no MLP outputs");
      for (int s = 0; s < d.n_springs; ++s) {
        const double* row = d.springs + 5 * (size_t)s;
        const int a = (int)row[0], b = (int)row[1];
        CLS_REQUIRE(a >= 0 && a < d.n_vertices && b >= 0 && b < d.n_vertices && a != b,
                    "spring endpoint out of range");
        h.sa.push_back(a);
        h.sb.push_back(b);
        h.len.push_back(row[2]);
        h.stiff.push_back(row[3] * p.stiffness_scale);
        h.coef.push_back(row[4]);
        int o = d.spring_output ? d.spring_output[s] : s;
        CLS_REQUIRE(o >= -1 && o < h.n_out, "spring_output index out of range");
        h.out.push_back(o);
      }
      h.n_layers = d.n_hidden_layers + 1;
      const int n_goal = (p.duplicate_v > 0 ? 2 : 0) + (p.duplicate_h > 0 ? 1 : 0) + (p.duplicate_c > 0 ? 1 : 0);
      h.pos_pad = round4(3 * h.n_v);
      h.n_c = h.pos_pad + p.n_sin_waves + n_goal;
      h.width[0] = h.n_c;
      h.full_cols[0] = p.n_sin_waves + 6 * h.n_v + 2 * p.duplicate_v + p.duplicate_h + p.duplicate_c;
      for (int l = 1; l < h.n_layers; ++l) {
        CLS_REQUIRE(d.hidden[l - 1] > 0, "hidden width must be > 0");
        h.width[l] = d.hidden[l - 1];
        h.full_cols[l] = d.hidden[l - 1];
      }
      h.width[h.n_layers] = h.n_out;
    }
    std::vector<int> er(env_robot, env_robot + n_envs);
    for (int e : er) CLS_REQUIRE(e >= 0 && e < n_robots, "env_robot index out of range");
    auto* s = new cls_sim;
    try {
      if (p.precision == 32) s->impl.reset(new SimImpl<float>(hr, er, p));
      else s->impl.reset(new SimImpl<double>(hr, er, p));
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
    return CLS_OK;
  } catch (const Fail& e) {
    g_create_error = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return CLS_ERR_INVALID;
  }
}

int cls_destroy(cls_sim* sim) {
  if (!sim) return CLS_ERR_INVALID;
  delete sim;
  return CLS_OK;
}

const char* cls_last_error(const cls_sim* sim) {
  if (!sim || !sim->impl) return cls::g_create_error.c_str();
  return sim->impl->err.c_str();
}

int cls_set_stream(cls_sim* sim, void* stream) {
  return guarded(sim, [&](cls::SimBase& b) { b.stream = (cudaStream_t)stream; });
}

int cls_get_sizes(const cls_sim* sim, int32_t* n_envs, int32_t* n_vertices_total, int32_t* max_steps) {
  if (!sim || !sim->impl) return CLS_ERR_INVALID;
  sim->impl->sizes(n_envs, n_vertices_total, max_steps);
  return CLS_OK;
}

int cls_get_layer_shape(const cls_sim* sim, int32_t robot, int32_t layer, int32_t* rows, int32_t* cols) {
  return guarded(const_cast<cls_sim*>(sim),
                 [&](cls::SimBase& b) { b.layer_shape(robot, layer, rows, cols); });
}

int cls_set_state(cls_sim* sim, const double* x0, const double* v0) {
  return guarded(sim, [&](cls::SimBase& b) { b.set_state(x0, v0); });
}

int cls_set_targets(cls_sim* sim, const double* tv, const double* th, const double* tc) {
  return guarded(sim, [&](cls::SimBase& b) { b.set_targets(tv, th, tc); });
}

int cls_set_weights(cls_sim* sim, int32_t robot, int32_t layer, const double* W, const double* b) {
  return guarded(sim, [&](cls::SimBase& s) { s.set_weights(robot, layer, W, b); });
}

int cls_get_weights(cls_sim* sim, int32_t robot, int32_t layer, double* W, double* b) {
  return guarded(sim, [&](cls::SimBase& s) { s.get_weights(robot, layer, W, b); });
}

int cls_get_grads(cls_sim* sim, int32_t robot, int32_t layer, double* gW, double* gb) {
  return guarded(sim, [&](cls::SimBase& s) { s.get_grads(robot, layer, gW, gb); });
}

int cls_forward(cls_sim* sim, int32_t steps) {
  return guarded(sim, [&](cls::SimBase& s) { s.forward(steps, false, false); });
}

int cls_forward_eval(cls_sim* sim, int32_t steps) {
  return guarded(sim, [&](cls::SimBase& s) { s.forward(steps, true, false); });
}

int cls_loss(cls_sim* sim, double* terms, double* env) {
  return guarded(sim, [&](cls::SimBase& s) { s.loss(terms, env); });
}

int cls_backward(cls_sim* sim) {
  return guarded(sim, [&](cls::SimBase& s) { s.backward(false); });
}

int cls_serve_reset_env(cls_sim* sim, int32_t env, const double* x0, const double* v0, const double* tv,
                        const double* th, const double* tc) {
  return guarded(sim, [&](cls::SimBase& s) { s.serve_reset_env(env, x0, v0, tv, th, tc); });
}
int cls_serve_forward(cls_sim* sim, const int32_t* windows, const int32_t* steps) {
  return guarded(sim, [&](cls::SimBase& s) { s.serve_forward(windows, steps); });
}
int cls_serve_backward(cls_sim* sim, const int32_t* windows, const int32_t* steps) {
  return guarded(sim, [&](cls::SimBase& s) { s.serve_backward(windows, steps); });
}
int cls_serve_loss(cls_sim* sim, const int32_t* steps, double* env) {
  return guarded(sim, [&](cls::SimBase& s) { s.serve_loss(steps, env); });
}
int cls_serve_env_state(cls_sim* sim, int32_t env, double* x, double* v) {
  return guarded(sim, [&](cls::SimBase& s) { s.serve_env_state(env, x, v); });
}

int cls_serve_tick(cls_sim* sim, int32_t tick_segments) {
  return guarded(sim, [&](cls::SimBase&) {
    CLS_REQUIRE(tick_segments >= 1, "tick_segments must be >= 1");
    sim->tick_segments = tick_segments;
    if (sim->sched) sim->sched->set_rounds(tick_segments);
  });
}

int cls_admit(cls_sim* sim, const cls_request* req, int64_t bytes_budget, int32_t* slot) {
  return guarded(sim, [&](cls::SimBase&) {
    CLS_REQUIRE(req != nullptr && slot != nullptr, "request and slot are required");
    *slot = cls::scheduler(sim).admit(req->id, req->robot, req->steps, req->grad != 0, req->x0, req->target_v,
                                      req->target_h, req->target_c, bytes_budget);
  });
}

int cls_poll(cls_sim* sim, uint64_t* done, int32_t capacity, int32_t* n_done, int32_t* n_active) {
  return guarded(sim, [&](cls::SimBase&) {
    CLS_REQUIRE(capacity >= 0 && (capacity == 0 || done != nullptr), "done needs capacity entries");
    cls::SlotScheduler& q = cls::scheduler(sim);
    q.poll();
    const int k = q.report(done, capacity);
    if (n_done) *n_done = k;
    if (n_active) *n_active = q.active();
  });
}

int cls_serve_result(cls_sim* sim, uint64_t id, int32_t* slot, double* loss_terms, double* final_x) {
  return guarded(sim, [&](cls::SimBase&) {
    const int s = cls::scheduler(sim).result(id, loss_terms, final_x);
    if (slot) *slot = s;
  });
}

int cls_serve_release(cls_sim* sim, uint64_t id) {
  return guarded(sim, [&](cls::SimBase&) { cls::scheduler(sim).release(id); });
}

int cls_simulate(cls_sim* sim, int32_t steps, double* loss) {
  return guarded(sim, [&](cls::SimBase& s) {
    s.forward(steps, false, false);
    double t8[8];
    s.loss(t8, nullptr);
    s.backward(false);
    if (loss) *loss = t8[0];
  });
}

int cls_simulate_per_env(cls_sim* sim, int32_t steps, double* loss) {
  return guarded(sim, [&](cls::SimBase& s) {
    s.forward(steps, false, true);
    double t8[8];
    s.loss(t8, nullptr);
    s.backward(true);
    if (loss) *loss = t8[0];
  });
}

int cls_adam_step(cls_sim* sim, int32_t iter, double* tns) {
  return guarded(sim, [&](cls::SimBase& s) { s.adam(iter, tns); });
}

int cls_clear_adam(cls_sim* sim) {
  return guarded(sim, [&](cls::SimBase& s) { s.clear_adam(); });
}

int cls_get_observables(cls_sim* sim, double* center, double* height, double* upper, double* rot) {
  return guarded(sim, [&](cls::SimBase& s) { s.observables(center, height, upper, rot); });
}

int cls_grad_buffers(cls_sim* sim, void** weight_grads, int64_t* n_weight, void** bias_grads,
                     int64_t* n_bias, int32_t* elem_bytes) {
  if (!weight_grads || !n_weight || !bias_grads || !n_bias || !elem_bytes) return CLS_ERR_INVALID;
  return guarded(sim, [&](cls::SimBase& s) {
    long long nw = 0, nb = 0;
    int e = 0;
    s.grad_buffers(weight_grads, &nw, bias_grads, &nb, &e);
    *n_weight = nw;
    *n_bias = nb;
    *elem_bytes = e;
  });
}

int cls_env_step(cls_sim* sim, int32_t t, const double* outputs, double* observation, double* center_height) {
  return guarded(sim, [&](cls::SimBase& s) { s.env_step(t, outputs, observation, center_height); });
}

int cls_serve_set_targets(cls_sim* sim, int32_t env, int32_t t_from, const double* tv, const double* th,
                          const double* tc) {
  return guarded(sim, [&](cls::SimBase& s) { s.env_set_targets(env, t_from, tv, th, tc); });
}

int cls_debug_gemm_starve(cls_sim* sim, int32_t starve, uint32_t wait_limit) {
  return guarded(sim, [&](cls::SimBase& s) { s.debug_gemm_starve(starve, wait_limit); });
}

int cls_set_loss_envs(cls_sim* sim, int32_t robot, int32_t n_envs) {
  return guarded(sim, [&](cls::SimBase& s) { s.set_loss_envs(robot, n_envs); });
}

int cls_set_loss_mask(cls_sim* sim, int32_t mask) {
  return guarded(sim, [&](cls::SimBase& s) { s.set_loss_mask(mask); });
}

int cls_get_targets(cls_sim* sim, double* tv, double* th, double* tc) {
  return guarded(sim, [&](cls::SimBase& s) { s.targets(tv, th, tc); });
}

int cls_get_trajectory(cls_sim* sim, double* x) {
  return guarded(sim, [&](cls::SimBase& s) { s.trajectory(x); });
}

int cls_get_final_state(cls_sim* sim, double* x, double* v) {
  return guarded(sim, [&](cls::SimBase& s) { s.final_state(x, v); });
}

int cls_get_state_grads(cls_sim* sim, double* gx0, double* gv0) {
  return guarded(sim, [&](cls::SimBase& s) { s.state_grads(gx0, gv0); });
}

int cls_synchronize(cls_sim* sim) {
  if (!sim || !sim->impl) return CLS_ERR_INVALID;
  int rc = CLS_OK;
  int g = guarded(sim, [&](cls::SimBase& s) { rc = s.synchronize(); });
  return g != CLS_OK ? g : rc;
}

int cls_weights_init(cls_sim* sim, uint64_t seed) {
  return guarded(sim, [&](cls::SimBase& s) { s.weights_init(seed); });
}

int cls_initialize_train(cls_sim* sim, int32_t iter, int32_t steps, uint64_t seed, double max_speed) {
  return guarded(sim, [&](cls::SimBase& s) { s.initialize_train(iter, steps, seed, max_speed); });
}

int cls_profile_enable(cls_sim* sim, int32_t on) {
  return guarded(sim, [&](cls::SimBase& s) { s.profile_enable(on != 0); });
}

int cls_profile_read(cls_sim* sim, double* ms, int64_t* launches, int32_t reset) {
  return guarded(sim, [&](cls::SimBase& s) {
    long long l[cls::PK_COUNT];
    s.profile_read(ms, l, reset != 0);
    if (launches)
      for (int k = 0; k < cls::PK_COUNT; ++k) launches[k] = l[k];
  });
}

// per-phase clock totals (32 slots); zeros unless built with CLS_PHASE_TIMERS
int cls_phase_read(cls_sim* sim, unsigned long long* out) {
  if (!out) return CLS_ERR_INVALID;
  return guarded(sim, [&](cls::SimBase& s) { s.phase_read(out); });
}

int cls_graph_capture(cls_sim* sim, int32_t steps, int32_t with_adam) {
  return guarded(sim, [&](cls::SimBase& s) { s.graph_capture(steps, with_adam != 0); });
}

int cls_graph_launch(cls_sim* sim, int32_t iter) {
  return guarded(sim, [&](cls::SimBase& s) { s.graph_launch(iter); });
}

int cls_set_controller_path(cls_sim* sim, int32_t path) {
  return guarded(sim, [&](cls::SimBase& s) { s.set_controller_path(path); });
}

int cls_controller_batched(const cls_sim* sim, int32_t* on) {
  if (!sim || !sim->impl || !on) return CLS_ERR_INVALID;
  *on = sim->impl->controller_batched() ? 1 : 0;
  return CLS_OK;
}

int cls_set_launch_shape(cls_sim* sim, int32_t threads_per_block, int32_t ctas_per_sm,
                         int32_t weights_shared) {
  return guarded(sim, [&](cls::SimBase& s) {
    s.set_launch_shape(threads_per_block, ctas_per_sm, weights_shared);
  });
}

int cls_get_launch_shape(const cls_sim* sim, int32_t* threads_per_block, int32_t* ctas_per_sm,
                         int32_t* weights_shared) {
  if (!sim || !sim->impl || !threads_per_block || !ctas_per_sm) return CLS_ERR_INVALID;
  int t = 0, c = 0, w = 0;
  sim->impl->launch_shape(&t, &c, &w);
  *threads_per_block = t;
  *ctas_per_sm = c;
  if (weights_shared) *weights_shared = w;
  return CLS_OK;
}

int cls_set_spring_tables(cls_sim* sim, int32_t mode) {
  return guarded(sim, [&](cls::SimBase& s) { s.set_spring_tables(mode); });
}

int cls_spring_tables(const cls_sim* sim, int32_t* on) {
  if (!sim || !sim->impl || !on) return CLS_ERR_INVALID;
  *on = sim->impl->spring_tables() ? 1 : 0;
  return CLS_OK;
}

int cls_autotune(cls_sim* sim, int32_t steps, int32_t repeats, cls_launch_shape* table,
                 int32_t max_entries, int32_t* n_entries) {
  if (max_entries < 0 || (max_entries > 0 && !table)) return CLS_ERR_INVALID;
  return guarded(sim, [&](cls::SimBase& s) {
    std::vector<cls_launch_shape> t;
    s.autotune(steps, repeats, t);
    for (int i = 0; i < (int)t.size() && i < max_entries; ++i) table[i] = t[i];
    if (n_entries) *n_entries = (int32_t)t.size();
  });
}

}  // extern "C"
