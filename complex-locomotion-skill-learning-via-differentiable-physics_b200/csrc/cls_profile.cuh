// cls_profile.cuh -- per-category CUDA-event timing of kernel launches on one
// stream.  Each timed launch is bracketed by a pair of events; collect()
// synchronises the stream and adds the elapsed times to the category totals.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace cls {

template <int NK>
struct EventProfile {
  bool on = false;
  std::vector<cudaEvent_t> ev;  // pairs (start, stop)
  std::vector<int> kind;
  size_t used = 0;
  double ms[NK] = {0};
  long long launches[NK] = {0};

  ~EventProfile() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }

  // Runs f (which enqueues work on `stream`), counted under `k` and, when
  // profiling is on, bracketed by events.  Returns the first CUDA error.
  template <typename F>
  cudaError_t run(int k, cudaStream_t stream, F&& f) {
    launches[k] += 1;
    if (!on) {
      f();
      return cudaSuccess;
    }
    if (used + 2 > ev.size()) {
      for (int q = 0; q < 64; ++q) {
        cudaEvent_t e;
        const cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        ev.push_back(e);
      }
    }
    cudaEvent_t a = ev[used], b = ev[used + 1];
    used += 2;
    kind.push_back(k);
    cudaError_t r = cudaEventRecord(a, stream);
    if (r != cudaSuccess) return r;
    f();
    return cudaEventRecord(b, stream);
  }

  cudaError_t collect(cudaStream_t stream) {
    if (used == 0) return cudaSuccess;
    cudaError_t r = cudaStreamSynchronize(stream);
    if (r != cudaSuccess) return r;
    for (size_t q = 0; q < kind.size(); ++q) {
      float t = 0;
      r = cudaEventElapsedTime(&t, ev[2 * q], ev[2 * q + 1]);
      if (r != cudaSuccess) return r;
      ms[kind[q]] += t;
    }
    kind.clear();
    used = 0;
    return cudaSuccess;
  }

  void read(double* out_ms, long long* out_launches, bool reset) {
    for (int k = 0; k < NK; ++k) {
      if (out_ms) out_ms[k] = ms[k];
      if (out_launches) out_launches[k] = launches[k];
    }
    if (reset)
      for (int k = 0; k < NK; ++k) { ms[k] = 0; launches[k] = 0; }
  }
};

}  // namespace cls
