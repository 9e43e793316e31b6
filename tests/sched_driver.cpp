// Test driver of the library's slot scheduler (csrc/ms_sched.h) on the CPU:
// a recording fake of the served handle, commands on stdin, one JSON object
// per line on stdout.  Built by tests/test_sched_cpu.py with g++.
//
//   sched_driver n_slots max_steps K rounds class_0 ... class_{n-1}
//   admit <id> <robot> <steps> <grad> <budget>   -> {"admit": id, "slot": s}
//   poll                                         -> launches, then {"done": [...], "active": a}
//   result <id>                                  -> {"result": id, "slot": s, "terms": [...], "x": [...]}
//   release <id> | rounds <n>                    -> {"ok": 1}
// Failures print {"error": "..."}.  A negative class marks slots whose
// robot entry other slots share (no gradient queries).  The fake's footprint is
// steps x (3 with gradients, else 1) + 1000 x slot class; its loss terms are
// k + 10 x slot + 0.001 x steps; its final positions are (slot, steps, k).
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "ms_sched.h"

namespace {

struct FakeOps final : cls::SlotOps {
  int n = 0, T = 0, K = 0;
  std::vector<int> cls_;
  std::vector<int> reset_steps;
  int n_slots() const override { return n; }
  int max_steps() const override { return T; }
  int checkpoint_every() const override { return K; }
  int slot_class(int s) const override { return cls_[s]; }
  int n_vertices(int) const override { return 2; }
  bool own_controller(int s) const override { return cls_[s] >= 0; }
  long long footprint(int s, int steps, bool grad) const override {
    return (long long)steps * (grad ? 3 : 1) + 1000LL * cls_[s];
  }
  void reset(int s, const double*, const double*, const double*, const double*) override {
    std::printf("{\"reset\": %d}\n", s);
  }
  void windows(const char* kind, const int* w, const int* st) {
    std::printf("{\"%s\": [", kind);
    bool first = true;
    for (int i = 0; i < n; ++i) {
      if (w[4 * i] >= w[4 * i + 1]) continue;
      std::printf("%s[%d, %d, %d, %d, %d, %d]", first ? "" : ", ", i, w[4 * i], w[4 * i + 1], w[4 * i + 2],
                  w[4 * i + 3], st[i]);
      first = false;
    }
    std::printf("]}\n");
  }
  void forward(const int* w, const int* st) override { windows("forward", w, st); }
  void backward(const int* w, const int* st) override { windows("backward", w, st); }
  void loss(const int* st, double* env) override {
    std::printf("{\"loss\": [");
    bool first = true;
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 8; ++k) env[(size_t)k * n + i] = st[i] > 0 ? k + 10.0 * i + 0.001 * st[i] : 0.0;
      if (st[i] > 0) {
        std::printf("%s[%d, %d]", first ? "" : ", ", i, st[i]);
        first = false;
      }
    }
    std::printf("]}\n");
  }
  void final_x(int s, double* x) override {
    for (int k = 0; k < 6; ++k) x[k] = k % 3 == 0 ? s : (k % 3 == 1 ? 7.0 : k);
  }
  void wait() override {}
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  FakeOps ops;
  ops.n = std::atoi(argv[1]);
  ops.T = std::atoi(argv[2]);
  ops.K = std::atoi(argv[3]);
  const int rounds = std::atoi(argv[4]);
  if (argc != 5 + ops.n) return 2;
  for (int i = 0; i < ops.n; ++i) ops.cls_.push_back(std::atoi(argv[5 + i]));
  cls::SlotScheduler q(ops, rounds);
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream in(line);
    std::string cmd;
    if (!(in >> cmd)) continue;
    try {
      if (cmd == "admit") {
        unsigned long long id;
        int robot, steps, grad;
        long long budget;
        in >> id >> robot >> steps >> grad >> budget;
        const int s = q.admit(id, robot, steps, grad != 0, nullptr, nullptr, nullptr, nullptr, budget);
        std::printf("{\"admit\": %llu, \"slot\": %d, \"used\": %lld}\n", id, s, q.used_bytes());
      } else if (cmd == "poll") {
        q.poll();
        uint64_t ids[256];
        const int k = q.report(ids, 256);
        std::printf("{\"done\": [");
        for (int i = 0; i < k; ++i) std::printf("%s%llu", i ? ", " : "", (unsigned long long)ids[i]);
        std::printf("], \"active\": %d, \"in_flight\": %d}\n", q.active(), q.in_flight() ? 1 : 0);
      } else if (cmd == "result") {
        unsigned long long id;
        in >> id;
        double terms[8], x[6];
        const int s = q.result(id, terms, x);
        std::printf("{\"result\": %llu, \"slot\": %d, \"terms\": [", id, s);
        for (int k = 0; k < 8; ++k) std::printf("%s%.6f", k ? ", " : "", terms[k]);
        std::printf("], \"x\": [");
        for (int k = 0; k < 6; ++k) std::printf("%s%.6f", k ? ", " : "", x[k]);
        std::printf("]}\n");
      } else if (cmd == "release") {
        unsigned long long id;
        in >> id;
        q.release(id);
        std::printf("{\"ok\": 1, \"used\": %lld}\n", q.used_bytes());
      } else if (cmd == "rounds") {
        int r;
        in >> r;
        q.set_rounds(r);
        std::printf("{\"ok\": 1}\n");
      } else {
        std::printf("{\"error\": \"unknown command\"}\n");
      }
    } catch (const std::exception& e) {
      std::printf("{\"error\": \"%s\"}\n", e.what());
    }
    std::fflush(stdout);
  }
  return 0;
}
