// ms_sched.h -- continuous-batching slot scheduler of a served mass-spring
// handle: the state machine behind cls_admit / cls_poll (host-only C++).
//
// The reference has no serving loop (it trains one batch at a time,
// multitask/diffphy_trainer.py:219-256).  Every env of a served handle is a
// slot with a controller of its own.  A request is admitted into a free slot
// of its robot class when its HBM footprint fits the caller's budget beside
// the requests already admitted; admission restarts that slot alone.  Work
// advances by ticks: a tick runs, in one launch each, a forward window of
// `rounds * K` substeps for every slot in its first pass, then `rounds`
// reverse segments (one launch per round) for every slot in its reverse pass.
// poll() completes the tick in flight and issues the next one, so the device
// works while the caller reads results and admits more requests.  A finished
// slot keeps its loss terms, final positions and (gradient queries) weight
// gradients until the caller releases it.
//
// The tick plan (window tables, loss at the end of a first pass, reverse
// segments counted down from the last) is the one serving.Pool issues, so
// both schedulers give the same launches for the same requests.
#pragma once
#include <algorithm>
#include <cstdint>
#include <deque>
#include <stdexcept>
#include <vector>

namespace cls {

// What the scheduler drives: a served handle (the runtime's adapter) or a
// recording fake (the CPU tests).
struct SlotOps {
  virtual ~SlotOps() = default;
  virtual int n_slots() const = 0;
  virtual int max_steps() const = 0;
  virtual int checkpoint_every() const = 0;
  virtual int slot_class(int slot) const = 0;     // slots of one class run the same robot
  virtual int n_vertices(int slot) const = 0;
  virtual bool own_controller(int slot) const = 0;  // no other env shares the slot's robot entry
  virtual long long footprint(int slot, int steps, bool grad) const = 0;
  virtual void reset(int slot, const double* x0, const double* tv, const double* th, const double* tc) = 0;
  virtual void forward(const int* windows, const int* steps) = 0;   // [n_slots][4], [n_slots]
  virtual void backward(const int* windows, const int* steps) = 0;
  virtual void loss(const int* steps, double* env) = 0;             // env: [8][n_slots]
  virtual void final_x(int slot, double* x) = 0;                    // [n_v][3]
  virtual void wait() = 0;                                          // the tick in flight is done
};

struct SchedError : std::runtime_error {
  explicit SchedError(const char* m) : std::runtime_error(m) {}
};

class SlotScheduler {
 public:
  static constexpr int kLossTerms = 8;
  enum Phase : int { FREE = 0, FWD, REV, DONE };

  SlotScheduler(SlotOps& ops, int rounds) : ops_(ops), rounds_(std::max(1, rounds)) {
    slots_.resize(ops.n_slots());
  }

  void set_rounds(int rounds) {
    if (in_flight_) throw SchedError("the tick length changes only with no tick in flight");
    rounds_ = std::max(1, rounds);
  }
  int rounds() const { return rounds_; }
  long long used_bytes() const { return used_bytes_; }
  long long substeps_done() const { return substeps_done_; }

  // Admits request `id` on a free slot of slot_class(robot_slot); returns the
  // slot, or -1 when no slot of the class is free or its footprint does not
  // fit `budget` (< 0: no limit).  x0 null: the caller's reset supplies the
  // robot's rest pose; targets null: zeros.
  int admit(uint64_t id, int robot_slot, int steps, bool grad, const double* x0, const double* tv,
            const double* th, const double* tc, long long budget) {
    const int n = (int)slots_.size();
    if (robot_slot < 0 || robot_slot >= n) throw SchedError("robot slot out of range");
    if (steps < 2 || steps > ops_.max_steps()) throw SchedError("steps must be in [2, max_steps]");
    for (const Slot& s : slots_)
      if (s.phase != FREE && s.id == id) throw SchedError("request id already admitted");
    const int cls = ops_.slot_class(robot_slot);
    int pick = -1;
    for (int i = 0; i < n && pick < 0; ++i)
      if (slots_[i].phase == FREE && ops_.slot_class(i) == cls) pick = i;
    if (pick < 0) return -1;
    if (grad && !ops_.own_controller(pick))
      throw SchedError("gradient queries need a slot whose robot entry (controller) no other env shares");
    const long long fp = ops_.footprint(pick, steps, grad);
    if (budget >= 0 && used_bytes_ + fp > budget) return -1;
    ops_.reset(pick, x0, tv, th, tc);
    Slot& s = slots_[pick];
    s = Slot();
    s.phase = FWD;
    s.id = id;
    s.steps = steps;
    s.grad = grad;
    s.bytes = fp;
    used_bytes_ += fp;
    return pick;
  }

  // Completes the tick in flight (if any), then issues the next one (if any
  // slot is active).  Finished requests are queued for report().
  void poll() {
    if (in_flight_) complete();
    launch();
  }

  // Up to `cap` ids of finished requests not reported yet.
  int report(uint64_t* ids, int cap) {
    int k = 0;
    while (k < cap && !finished_.empty()) {
      ids[k++] = finished_.front();
      finished_.pop_front();
    }
    return k;
  }
  int unreported() const { return (int)finished_.size(); }

  int active() const {
    int a = 0;
    for (const Slot& s : slots_) a += (s.phase == FWD || s.phase == REV);
    return a;
  }
  bool in_flight() const { return in_flight_; }

  // Slot, loss terms (total, velocity, height, pose, rotation, weight,
  // actuation, crawl) and final positions of finished request `id`.
  int result(uint64_t id, double* terms, double* final_x) const {
    const int i = find(id);
    const Slot& s = slots_[i];
    if (s.phase != DONE) throw SchedError("the request has not finished");
    if (terms) std::copy(s.terms, s.terms + kLossTerms, terms);
    if (final_x) std::copy(s.fx.begin(), s.fx.end(), final_x);
    return i;
  }

  // Frees the slot of a finished request (its footprint leaves the budget).
  void release(uint64_t id) {
    const int i = find(id);
    Slot& s = slots_[i];
    if (s.phase != DONE) throw SchedError("only finished requests are released");
    used_bytes_ -= s.bytes;
    s = Slot();
  }

  Phase phase(int slot) const { return slots_.at(slot).phase; }

 private:
  struct Slot {
    Phase phase = FREE;
    uint64_t id = 0;
    int steps = 0;
    bool grad = false;
    int pos = 0;       // first pass: next substep to run
    int seg = 0;       // reverse pass: next segment to run
    long long bytes = 0;
    double terms[kLossTerms] = {0};
    std::vector<double> fx;
  };

  int find(uint64_t id) const {
    for (size_t i = 0; i < slots_.size(); ++i)
      if (slots_[i].phase != FREE && slots_[i].id == id) return (int)i;
    throw SchedError("unknown request id");
  }

  std::vector<int> steps_table() const {
    std::vector<int> st(slots_.size(), 2);
    for (size_t i = 0; i < slots_.size(); ++i)
      if (slots_[i].phase == FWD || slots_[i].phase == REV) st[i] = slots_[i].steps;
    return st;
  }

  void launch() {
    const int n = (int)slots_.size(), K = ops_.checkpoint_every();
    std::vector<int> st = steps_table();
    fw_.assign((size_t)4 * n, 0);
    bool any_f = false;
    for (int i = 0; i < n; ++i) {
      const Slot& s = slots_[i];
      if (s.phase != FWD) continue;
      const int t0 = s.pos, t_last = s.steps - 1;   // the first pass runs substeps [0, steps - 1)
      fw_[4 * i] = t0;
      fw_[4 * i + 1] = std::min(t0 + rounds_ * K, t_last);
      fw_[4 * i + 2] = t0 / K;
      any_f = true;
    }
    if (any_f) ops_.forward(fw_.data(), st.data());
    bool any_b = false;
    std::vector<int> bw((size_t)4 * n);
    for (int r = 0; r < rounds_; ++r) {
      std::fill(bw.begin(), bw.end(), 0);
      bool round_any = false;
      for (int i = 0; i < n; ++i) {
        const Slot& s = slots_[i];
        if (s.phase != REV || s.seg - r < 0) continue;
        const int t_last = s.steps - 1, n_seg = (t_last + K - 1) / K, seg = s.seg - r;
        bw[4 * i] = seg * K;
        bw[4 * i + 1] = std::min(seg * K + K, t_last);
        bw[4 * i + 2] = seg;
        bw[4 * i + 3] = seg == n_seg - 1 ? 1 : 0;
        round_any = true;
      }
      if (!round_any) break;
      ops_.backward(bw.data(), st.data());
      any_b = true;
    }
    in_flight_ = any_f || any_b;
    if (in_flight_) plan_steps_ = st;
  }

  void complete() {
    ops_.wait();
    in_flight_ = false;
    const int n = (int)slots_.size(), K = ops_.checkpoint_every();
    std::vector<int> fwd_finished;
    for (int i = 0; i < n; ++i) {
      Slot& s = slots_[i];
      if (s.phase == FWD && fw_[4 * i] < fw_[4 * i + 1]) {
        substeps_done_ += fw_[4 * i + 1] - fw_[4 * i];
        s.pos = fw_[4 * i + 1];
        if (s.pos >= s.steps - 1) fwd_finished.push_back(i);
      } else if (s.phase == REV) {
        s.seg -= rounds_;
      }
    }
    if (!fwd_finished.empty()) {
      std::vector<int> lsteps(n, 0);
      for (int i : fwd_finished) lsteps[i] = plan_steps_[i];
      std::vector<double> env((size_t)kLossTerms * n);
      ops_.loss(lsteps.data(), env.data());
      for (int i : fwd_finished) {
        Slot& s = slots_[i];
        for (int k = 0; k < kLossTerms; ++k) s.terms[k] = env[(size_t)k * n + i];
        s.fx.assign((size_t)3 * ops_.n_vertices(i), 0.0);
        ops_.final_x(i, s.fx.data());
        if (s.grad) {
          s.phase = REV;
          s.seg = (s.steps - 1 + K - 1) / K - 1;
        } else {
          finish(i);
        }
      }
    }
    for (int i = 0; i < n; ++i)
      if (slots_[i].phase == REV && slots_[i].seg < 0) finish(i);
  }

  void finish(int i) {
    slots_[i].phase = DONE;
    finished_.push_back(slots_[i].id);
  }

  SlotOps& ops_;
  int rounds_;
  std::vector<Slot> slots_;
  std::vector<int> fw_, plan_steps_;
  std::deque<uint64_t> finished_;
  long long used_bytes_ = 0, substeps_done_ = 0;
  bool in_flight_ = false;
};

}  // namespace cls
