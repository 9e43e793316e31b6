// noalloc.cu -- cls_ms_advance_noalloc: mass-spring substeps that allocate no
// memory at all.
//
// Who needs this: callers that are not allowed to allocate device memory --
// code running under a fixed device-memory budget owned by someone else (a
// game or robotics runtime with its own allocator, a serving process whose
// memory pool is pre-sized), or code that must not create allocations while a
// larger system is capturing its own work.  cls_create allocates its buffers
// with cudaMalloc, so such callers cannot use a cls_sim handle.  This entry
// point takes every input and output as a caller-owned device pointer and keeps
// its one piece of scratch -- the per-vertex velocity increment v_inc that the
// spring forces accumulate into -- in a fixed array that is part of the
// library image.
//
// Limits and sharing rules:
//   * the scratch holds kScratchFloats floats (2^21 = 8 MiB): calls need
//     n_envs * n_vertices * 3 <= kScratchFloats and are rejected otherwise;
//   * every GPU that loads the library holds that 8 MiB until the process ends;
//   * every call, on every stream, uses the same array: calls that overlap on
//     the GPU race with each other and give wrong results; serialise them;
//   * each call clears the part it uses before the first substep, so nothing
//     left from an earlier call leaks into the result;
//   * a __device__ array's address belongs to a CUDA context, so the first
//     call in each context (the runtime's primary context of a device, or a
//     context the caller created and made current with the driver API) looks
//     up the array's device address (cudaGetSymbolAddress) with that context
//     current and keeps it keyed by the context's unique id (cuCtxGetId: ids
//     are never reused, so a context created after cudaDeviceReset or
//     cuCtxDestroy gets a fresh lookup); make that first call before any
//     stream capture in that context;
//   * spring endpoints must lie in [0, n_vertices); a spring whose endpoint
//     does not is skipped (it exerts no force), so a bad table never reads or
//     writes outside the env's rows;
//   * a CUDA error already pending when the call starts (from the caller's
//     earlier work) is left in place and reported as CLS_ERR_CUDA without
//     launching anything.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/cls_b200.h"
#include "ms_kernels.cuh"

namespace {

constexpr long long kScratchFloats = 1LL << 21;
constexpr int kMaxContexts = 64;

// v_inc scratch ([env][vertex][3]); in host code this name is only a handle
// for cudaGetSymbolAddress, never a usable address
static __device__ __align__(256) float g_vinc_scratch[kScratchFloats];

// the scratch's address per CUDA context, keyed by the context's unique id
struct ScratchEntry {
  unsigned long long ctx_id;
  void* addr;
};
ScratchEntry g_scratch[kMaxContexts] = {};
int g_scratch_used = 0, g_scratch_next = 0;
std::mutex g_scratch_mutex;

// driver entry points, resolved through the runtime so that the library does
// not link libcuda (it must load on machines without a driver)
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

bool resolve_driver_calls() {
  if (g_ctx_get_current && g_ctx_get_id) return true;
  void* f0 = nullptr;
  void* f1 = nullptr;
  cudaDriverEntryPointQueryResult q0, q1;
  if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
      q0 != cudaDriverEntryPointSuccess || !f0)
    return false;
  if (cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
      q1 != cudaDriverEntryPointSuccess || !f1)
    return false;
  g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
  g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
  return true;
}

// id of the current context (0 when none is current)
unsigned long long current_ctx_id() {
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (g_ctx_get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// The scratch's device address in the current context; on the first call in a
// context, cudaGetSymbolAddress (which also makes the device's primary context
// current when no context is) resolves it with that context current.
cudaError_t scratch_address(float** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!resolve_driver_calls()) return cudaErrorNotSupported;
  unsigned long long id = current_ctx_id();
  if (id) {
    for (int i = 0; i < g_scratch_used; ++i)
      if (g_scratch[i].ctx_id == id) {
        *out = static_cast<float*>(g_scratch[i].addr);
        return cudaSuccess;
      }
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_vinc_scratch);
  if (e != cudaSuccess) return e;
  if (!p) return cudaErrorInvalidSymbol;
  if (!id) id = current_ctx_id();   // the lookup made the primary context current
  if (id) {
    int slot = g_scratch_used < kMaxContexts ? g_scratch_used++ : g_scratch_next;
    if (g_scratch_used == kMaxContexts) g_scratch_next = (slot + 1) % kMaxContexts;
    g_scratch[slot] = ScratchEntry{id, p};
  }
  *out = static_cast<float*>(p);
  return cudaSuccess;
}

void set_message(const cls_noalloc_advance* a, const char* msg) {
  if (a && a->error_message && a->error_capacity > 0)
    snprintf(a->error_message, (size_t)a->error_capacity, "%s", msg);
}

__global__ void na_clear(float* __restrict__ s, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    s[i] = 0.f;
}

// apply_spring_force (solver_mass_spring.py:86-105): one thread per (env,
// spring), impulses scattered into v_inc with atomics as the reference does
__global__ void na_spring(cls_noalloc_advance a, float* __restrict__ vinc) {
  const long long total = (long long)a.n_envs * a.n_springs;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q / a.n_springs), s = (int)(q % a.n_springs);
    const int ia = a.spring_a[s], ib = a.spring_b[s];
    if (ia < 0 || ia >= a.n_vertices || ib < 0 || ib >= a.n_vertices) continue;
    const float* xe = a.x + (size_t)e * a.n_vertices * 3;
    const float* ve = a.v + (size_t)e * a.n_vertices * 3;
    cls::V4<float> xa, xb, va, vb;
    xa.x = xe[3 * ia]; xa.y = xe[3 * ia + 1]; xa.z = xe[3 * ia + 2]; xa.w = 0;
    xb.x = xe[3 * ib]; xb.y = xe[3 * ib + 1]; xb.z = xe[3 * ib + 2]; xb.w = 0;
    va.x = ve[3 * ia]; va.y = ve[3 * ia + 1]; va.z = ve[3 * ia + 2]; va.w = 0;
    vb.x = ve[3 * ib]; vb.y = ve[3 * ib + 1]; vb.z = ve[3 * ib + 2]; vb.w = 0;
    float imp[3];
    cls::spring_impulse<float>(xa, xb, va, vb, a.rest_length[s], a.stiffness[s], a.actuation_coef[s],
                               a.actuation[(size_t)e * a.n_springs + s], a.dt, a.dashpot_damping, imp);
    float* vi = vinc + (size_t)e * a.n_vertices * 3;
    for (int d = 0; d < 3; ++d) {
      atomicAdd(vi + 3 * ia + d, -imp[d]);
      atomicAdd(vi + 3 * ib + d, imp[d]);
    }
  }
}

// advance_toi (solver_mass_spring.py:117-148) in place; consumes v_inc and
// leaves it zero for the next substep
__global__ void na_advance(cls_noalloc_advance a, float drag_s, float* __restrict__ vinc) {
  const long long total = (long long)a.n_envs * a.n_vertices;
  cls::MsArgs<float> p;
  p.dt = a.dt;
  p.gravity = a.gravity;
  p.ground = a.ground_height;
  p.drag_s = drag_s;
  p.friction = a.friction;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    float* xq = a.x + 3 * q;
    float* vq = a.v + 3 * q;
    float* iq = vinc + 3 * q;
    cls::V4<float> x, v, vi;
    x.x = xq[0]; x.y = xq[1]; x.z = xq[2]; x.w = 0;
    v.x = vq[0]; v.y = vq[1]; v.z = vq[2]; v.w = 0;
    vi.x = iq[0]; vi.y = iq[1]; vi.z = iq[2]; vi.w = 0;
    cls::advance_vertex<float>(p, x, v, vi);
    xq[0] = x.x; xq[1] = x.y; xq[2] = x.z;
    vq[0] = v.x; vq[1] = v.y; vq[2] = v.z;
    iq[0] = 0.f; iq[1] = 0.f; iq[2] = 0.f;
  }
}

int grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return g < 1 ? 1 : (int)g;
}

}  // namespace

extern "C" int cls_ms_advance_noalloc(const cls_noalloc_advance* a, void* stream) {
  if (!a) return CLS_ERR_INVALID;
  if (a->n_envs <= 0 || a->n_vertices <= 0 || a->n_springs < 0 || a->n_substeps < 0 || !a->x ||
      !a->v || (a->n_springs > 0 && (!a->spring_a || !a->spring_b || !a->rest_length ||
                                     !a->stiffness || !a->actuation_coef || !a->actuation))) {
    set_message(a, "cls_ms_advance_noalloc: missing pointer or non-positive size");
    return CLS_ERR_INVALID;
  }
  const long long need = (long long)a->n_envs * a->n_vertices * 3;
  if (need > kScratchFloats) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "cls_ms_advance_noalloc: n_envs * n_vertices * 3 = %lld exceeds the fixed scratch of "
             "%lld floats",
             need, kScratchFloats);
    set_message(a, msg);
    return CLS_ERR_INVALID;
  }
  // an error left by the caller's earlier work stays pending for the caller
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "cls_ms_advance_noalloc: a CUDA error from earlier work is pending (%s); nothing "
             "launched",
             cudaGetErrorName(pending));
    set_message(a, msg);
    return CLS_ERR_CUDA;
  }
  float* scratch = nullptr;
  const cudaError_t se = scratch_address(&scratch);
  if (se != cudaSuccess) {
    set_message(a, cudaGetErrorString(se));
    return CLS_ERR_CUDA;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float drag_s = (float)exp(-(double)a->dt * (double)a->drag_damping);
  na_clear<<<grid_for(need), 256, 0, s>>>(scratch, need);
  for (int step = 0; step < a->n_substeps; ++step) {
    if (a->n_springs > 0)
      na_spring<<<grid_for((long long)a->n_envs * a->n_springs), 256, 0, s>>>(*a, scratch);
    na_advance<<<grid_for((long long)a->n_envs * a->n_vertices), 256, 0, s>>>(*a, drag_s, scratch);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_message(a, cudaGetErrorString(e));
    return CLS_ERR_CUDA;
  }
  return CLS_OK;
}
