// cls_common.cuh -- shared device types and helpers for the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cls {

constexpr int kMaxLayers = 5;   // weight layers (hidden layers + output)

enum Act : int { ACT_SIN = 0, ACT_TANH = 1 };
enum LossBit : int {
  LOSS_VELOCITY = 1, LOSS_HEIGHT = 2, LOSS_POSE = 4,
  LOSS_ACTUATION = 8, LOSS_ROTATION = 16, LOSS_CRAWL = 32
};
// slots of the per-env loss record, in the reference's loss_dict order
// (multitask/taichi_env.py:82-88), total excluded
enum LossSlot : int { LS_VEL = 0, LS_HEIGHT = 1, LS_POSE = 2, LS_ROT = 3, LS_WEIGHT = 4,
                      LS_ACT = 5, LS_CRAWL = 6, LS_COUNT = 7 };

// error bits written to the device status word
enum ErrBit : int { ERR_NONFINITE = 1, ERR_SMEM = 2, ERR_CONFIG = 4, ERR_TIMEOUT = 8 };

// 4-wide vector, 16 B (float) / 32 B (double) aligned, for vectorised state I/O
template <typename R>
struct alignas(4 * sizeof(R)) V4 {
  R x, y, z, w;
};

// read-only (non-coherent) vector load
template <typename R> __device__ __forceinline__ V4<R> ldg4(const V4<R>* p);
template <> __device__ __forceinline__ V4<float> ldg4<float>(const V4<float>* p) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  V4<float> r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = v.w;
  return r;
}
template <> __device__ __forceinline__ V4<double> ldg4<double>(const V4<double>* p) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
  V4<double> r; r.x = a.x; r.y = a.y; r.z = b.x; r.w = b.y;
  return r;
}

// L2 eviction-priority policies (PTX createpolicy).  Controller weights are
// streamed once per substep and pass -- far more bytes than L2 holds -- so they
// are loaded evict_first; the spring incidence tables are re-read every
// substep and are loaded evict_last so the weight stream does not evict them.
__device__ __forceinline__ unsigned long long policy_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long policy_evict_last() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

template <typename R> __device__ __forceinline__ V4<R> ldg4_hint(const V4<R>* p, unsigned long long pol);
template <> __device__ __forceinline__ V4<float> ldg4_hint<float>(const V4<float>* p, unsigned long long pol) {
  V4<float> r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
               : "l"(p), "l"(pol));
  return r;
}
template <> __device__ __forceinline__ V4<double> ldg4_hint<double>(const V4<double>* p, unsigned long long pol) {
  V4<double> r;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
               : "=d"(r.x), "=d"(r.y)
               : "l"(p), "l"(pol));
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
               : "=d"(r.z), "=d"(r.w)
               : "l"(reinterpret_cast<const double*>(p) + 2), "l"(pol));
  return r;
}
__device__ __forceinline__ int4 ldg_i4_hint(const int4* p, unsigned long long pol) {
  int4 r;
  asm volatile("ld.global.nc.L2::cache_hint.v4.s32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p), "l"(pol));
  return r;
}

template <typename R>
__device__ __forceinline__ R comp(const V4<R>& v, int d) {
  return d == 0 ? v.x : (d == 1 ? v.y : v.z);
}

template <typename R> __device__ __forceinline__ R dsqrt(R x);
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }

// Spring-geometry helpers.  FP32 uses the hardware reciprocal square root
// (rsqrtf, <= 2 ulp) and the correctly rounded reciprocal (__frcp_rn) instead
// of IEEE sqrt / division sequences; FP64 -- the precision-check build -- keeps
// exact sqrt and division.
template <typename R> __device__ __forceinline__ R rsqrt_s(R x);
template <> __device__ __forceinline__ float rsqrt_s<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double rsqrt_s<double>(double x) { return 1.0 / sqrt(x); }
template <typename R> __device__ __forceinline__ R rcp_s(R x);
template <> __device__ __forceinline__ float rcp_s<float>(float x) { return __frcp_rn(x); }
template <> __device__ __forceinline__ double rcp_s<double>(double x) { return 1.0 / x; }
template <typename R> __device__ __forceinline__ R sqrt_s(R x);
template <> __device__ __forceinline__ float sqrt_s<float>(float x) { return x * rsqrtf(x); }
template <> __device__ __forceinline__ double sqrt_s<double>(double x) { return sqrt(x); }

template <typename R> __device__ __forceinline__ R dsin(R x);
template <> __device__ __forceinline__ float dsin<float>(float x) { return sinf(x); }
template <> __device__ __forceinline__ double dsin<double>(double x) { return sin(x); }
template <typename R> __device__ __forceinline__ R dcos(R x);
template <> __device__ __forceinline__ float dcos<float>(float x) { return cosf(x); }
template <> __device__ __forceinline__ double dcos<double>(double x) { return cos(x); }
template <typename R> __device__ __forceinline__ R dtanh(R x);
template <> __device__ __forceinline__ float dtanh<float>(float x) { return tanhf(x); }
template <> __device__ __forceinline__ double dtanh<double>(double x) { return tanh(x); }
template <typename R> __device__ __forceinline__ R datan2(R y, R x);
template <> __device__ __forceinline__ float datan2<float>(float y, float x) { return atan2f(y, x); }
template <> __device__ __forceinline__ double datan2<double>(double y, double x) { return atan2(y, x); }
template <typename R> __device__ __forceinline__ R dabs(R x);
template <> __device__ __forceinline__ float dabs<float>(float x) { return fabsf(x); }
template <> __device__ __forceinline__ double dabs<double>(double x) { return fabs(x); }
template <typename R> __device__ __forceinline__ R dpow_half(R x);
template <> __device__ __forceinline__ float dpow_half<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double dpow_half<double>(double x) { return sqrt(x); }

// activation and its derivative, evaluated at the pre-activation u = z + b
template <typename R>
__device__ __forceinline__ R act_f(int kind, R u) {
  return kind == ACT_TANH ? dtanh<R>(u) : dsin<R>(u);
}
template <typename R>
__device__ __forceinline__ R act_d(int kind, R u) {
  if (kind == ACT_TANH) {
    R y = dtanh<R>(u);
    return R(1) - y * y;
  }
  return dcos<R>(u);
}

template <typename R>
__device__ __forceinline__ bool finite(R x) {
  return isfinite(x);
}

// deterministic block reduction (fixed tree for a fixed blockDim); `red` must
// hold >= 32 elements; every thread receives the result
template <typename T, typename Op>
__device__ __forceinline__ T block_reduce(T v, T* red, Op op) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    T w = (lane < nw) ? red[lane] : red[0];
    // lanes >= nw hold a duplicate of red[0]; the tree below only combines
    // lanes < nw because the identity is applied through a mask
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      T other = __shfl_down_sync(0xffffffffu, w, o);
      if (lane + o < nw) w = op(w, other);
    }
    if (lane == 0) red[0] = w;
  }
  __syncthreads();
  T r = red[0];
  __syncthreads();
  return r;
}

struct OpSum {
  template <typename T> __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};

}  // namespace cls
