// umma_gemm.cuh -- tcgen05 (5th-generation tensor core) building blocks for
// FP32-accurate GEMM tiles: C(i, j) = sum_k A(i, k) B(j, k) with FP32 operands
// split into TF32 high and low parts ("3xTF32": a_lo b_hi + a_hi b_lo +
// a_hi b_hi, about FP32 accuracy) and the FP32 accumulator in tensor memory.
// Operands arrive pre-split in global memory in the MMA's 128-byte-swizzled
// K-major layout (SplitTiles) and are streamed into shared memory with bulk
// copies completing on mbarriers (tile_gemm_bulk).  Descriptor and
// instruction-descriptor bit layouts follow the PTX ISA's tcgen05 matrix
// descriptors (as CUTLASS's cute/arch/mma_sm100_desc.hpp encodes them).
//
// Tensor memory: TN columns rounded up to a power of two (>= 32).  Callers
// keep TN <= 128 and at least TN * 456 bytes of shared memory per CTA, so the
// CTAs that fit on one SM never ask for more than its 512 columns (an
// allocation that cannot be satisfied would wait).
//
// Every wait is bounded: on a timeout the tile reports failure and returns
// after freeing its tensor memory.
#pragma once
#include <cstdint>

namespace cls {
namespace umma {

constexpr int TM = 128;        // output rows per tile (MMA M)
constexpr int TK = 32;         // K values per stage (4 MMA K-steps of 8)
constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// shared-memory matrix descriptor of the 128-byte swizzled K-major layout:
// start address (16-byte units), rows of 128 bytes, 8-row atoms of 1024 bytes
// (stride byte offset), leading byte offset unused (1), descriptor version 1,
// base offset 0, layout type 2; a K step inside the atom advances the start
// address
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

// instruction descriptor: FP32 accumulator (bits 4-5 = 1), TF32 A and B (bits
// 7-9 and 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24
__host__ __device__ constexpr uint32_t instr_desc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
      "}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(phase)
      : "memory");
  return ok != 0;
}

// bounded wait for the phase (at most `limit` polls); false on timeout
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, unsigned limit = kWaitLimit) {
  for (unsigned it = 0; it < limit; ++it)
    if (mbar_try_wait(mbar, phase)) return true;
  return false;
}

// Wait policy of a tile: the poll limit of every wait (0: kWaitLimit) and the
// self-test mode `starve`, in which the producer issues no bulk copies and
// the MMA issuer no MMAs, so the issuer's first wait for operands runs out
// with nothing in flight and the tile takes its timeout path (status bit,
// tensor memory freed, no epilogue).
struct WaitPolicy {
  unsigned limit;
  int starve;
};

__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// a CTA that will allocate no more tensor memory lets waiting CTAs in
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// 32 lanes x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float v[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void split4(const float4& v4, uint4& hi, uint4& lo) {
  const float v[4] = {v4.x, v4.y, v4.z, v4.w};
  uint32_t* h = &hi.x;
  uint32_t* l = &lo.x;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    h[u] = tf32_bits(v[u]);
    l[u] = tf32_bits(v[u] - __uint_as_float(h[u]));
  }
}

// ------------------------------------------------------ pre-split operand tiles
// Operands of tile_gemm_bulk live in global memory already split and laid out
// exactly like one shared-memory stage: for a matrix of R rows (tile height
// TR) and K columns, the block of rows [rt TR, rt TR + TR) and columns
// [32 kt, 32 kt + 32) is 2 * 32 * TR contiguous floats, the TF32 high part
// then the low part.  Within a part each row is one 128-byte line (32 TF32
// values) and the 16-byte chunks of row r are XOR-permuted by r mod 8 -- the
// MMA's 128-byte swizzled K-major layout (the canonical SWIZZLE_128B form of
// the tcgen05 shared-memory descriptor), whose 8-row atoms (1024 bytes) the
// tensor core reads without bank conflicts: element (r, k) sits at float
// r * 32 + 4 ((k % 32) / 4 xor r % 8) + k % 4.  Blocks are ordered (rt, kt)
// with kt fastest, 1024-byte aligned.  Entries never written (rows >= R,
// columns >= K) stay zero.  The producers of the operands (the step kernels,
// the previous layer's epilogue, the weight packing) write this form, so a
// GEMM stage is two bulk copies.
struct SplitTiles {
  float* p;
  int tr, nkt;
  __device__ __forceinline__ size_t index(int r, int k) const {
    const int kk = k & 31, rr = r % tr;
    return ((size_t)(r / tr) * nkt + (k >> 5)) * (size_t)(64 * tr) + (size_t)rr * 32 +
           (size_t)((((kk >> 2) ^ (rr & 7))) << 2) + (kk & 3);
  }
  __device__ __forceinline__ void store(int r, int k, float v) const {
    const size_t o = index(r, k);
    const uint32_t h = tf32_bits(v);
    p[o] = __uint_as_float(h);
    p[o + 32 * tr] = __uint_as_float(tf32_bits(v - __uint_as_float(h)));
  }
  // the same with the tile height TR (== tr) known at compile time
  template <int TR>
  __device__ __forceinline__ void store_tr(int r, int k, float v) const {
    const int kk = k & 31, rr = r % TR;
    const size_t o = ((size_t)(r / TR) * nkt + (k >> 5)) * (size_t)(64 * TR) + (size_t)rr * 32 +
                     (size_t)((((kk >> 2) ^ (rr & 7))) << 2) + (kk & 3);
    const uint32_t h = tf32_bits(v);
    p[o] = __uint_as_float(h);
    p[o + 32 * TR] = __uint_as_float(tf32_bits(v - __uint_as_float(h)));
  }
  // four consecutive columns k .. k + 3 (k a multiple of 4)
  __device__ __forceinline__ void store4(int r, int k, const float4& v) const {
    const size_t o = index(r, k);
    uint4 hi, lo;
    split4(v, hi, lo);
    *reinterpret_cast<uint4*>(p + o) = hi;
    *reinterpret_cast<uint4*>(p + o + 32 * tr) = lo;
  }
};

__host__ __device__ constexpr size_t split_tiles_floats(int rows, int tr, int k) {
  return (size_t)((rows + tr - 1) / tr) * (size_t)((k + 31) / 32) * (size_t)(64 * tr);
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

constexpr int kBulkThreads = 128;  // 4 warps: warp w reads accumulator lanes [32 w, 32 w + 32)
constexpr int kMaxStages = 6;

template <int TN, int S>
struct BulkShape {
  static_assert(TN % 16 == 0 && TN >= 16 && TN <= 128, "MMA N: multiple of 16 in [16, 128]");
  static_assert(S >= 2 && S <= kMaxStages, "stages");
  static constexpr int kCols = TN <= 32 ? 32 : (TN <= 64 ? 64 : 128);
  static constexpr uint32_t kABytes = 2 * TK * TM * 4;  // hi + lo of one 128 x 32 block
  static constexpr uint32_t kBBytes = 2 * TK * TN * 4;
  static constexpr uint32_t kStageBytes = kABytes + kBBytes;
  static constexpr size_t kRing = (size_t)S * kStageBytes;
  static constexpr size_t kSmemBytes = kRing > (size_t)kCols * 456 ? kRing : (size_t)kCols * 456;
};

struct BulkShared {
  uint64_t full[kMaxStages];   // stage filled (bulk copies' bytes arrived)
  uint64_t empty[kMaxStages];  // stage consumed (its MMAs completed)
  uint64_t done;               // every MMA of the tile completed
  uint32_t tmem_base;
  int timed_out;
};

// One 128 x TN tile, C(i, j) = sum_k A(i, k) B(j, k) over the whole K range:
// `a_blocks` / `b_blocks` point at block (rt, 0) / (nt, 0) of SplitTiles
// operands with nkt K-blocks each (tile heights 128 / TN).  Thread 0 fills an
// S-stage ring with bulk copies, thread 32 issues the MMAs (3 per K-step of
// 8: lo*hi, hi*lo, hi*hi) and commits each stage back to the producer.  The
// accumulator is then staged through the (idle) ring as a row-major
// 128 x TN tile, C(i, j) at cs[i * ld + j], and epi(cs, ld) writes it out
// with every thread of the CTA (so its global stores can run along rows).
// kBulkThreads threads.  Returns false on a timeout (epi is not called then).
template <int TN, int S, typename Epi>
__device__ bool tile_gemm_bulk(float* smem, BulkShared& bs, const float* a_blocks, const float* b_blocks,
                               int nkt, Epi epi, WaitPolicy wp = WaitPolicy{0u, 0}) {
  using Sh = BulkShape<TN, S>;
  const unsigned lim = wp.limit ? wp.limit : kWaitLimit;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t full0 = smem_u32(&bs.full[0]), empty0 = smem_u32(&bs.empty[0]), done = smem_u32(&bs.done);
  const uint32_t ring = smem_u32(smem);
  if (warp == 0) tmem_alloc(smem_u32(&bs.tmem_base), Sh::kCols);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done, 1);
    bs.timed_out = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = bs.tmem_base;
  constexpr uint32_t idesc = instr_desc_tf32(TM, TN);
  if (tid == 0 && !wp.starve) {
    // producer: two bulk copies per stage
    for (int kt = 0; kt < nkt; ++kt) {
      const int s = kt % S;
      if (kt >= S && !mbar_wait(empty0 + 8 * s, ((kt / S) - 1) & 1, lim)) { bs.timed_out = 1; break; }
      const uint32_t st = ring + (uint32_t)s * Sh::kStageBytes;
      mbar_arrive_expect_tx(full0 + 8 * s, Sh::kStageBytes);
      bulk_g2s(st, a_blocks + (size_t)kt * (2 * TK * TM), Sh::kABytes, full0 + 8 * s);
      bulk_g2s(st + Sh::kABytes, b_blocks + (size_t)kt * (2 * TK * TN), Sh::kBBytes, full0 + 8 * s);
    }
  } else if (tid == 32) {
    // MMA issuer
    for (int kt = 0; kt < nkt; ++kt) {
      const int s = kt % S;
      if (!mbar_wait(full0 + 8 * s, (kt / S) & 1, lim)) { bs.timed_out = 1; break; }
      tc_fence_after();
      const uint32_t a_hi = ring + (uint32_t)s * Sh::kStageBytes, a_lo = a_hi + TK * TM * 4;
      const uint32_t b_hi = a_hi + Sh::kABytes, b_lo = b_hi + TK * TN * 4;
#pragma unroll
      for (int ks = 0; ks < TK / 8; ++ks) {
        // K step ks: bytes [32 ks, 32 ks + 32) of every 128-byte row
        const uint32_t o = 32 * ks;
        const uint64_t dah = smem_desc_sw128(a_hi + o), dal = smem_desc_sw128(a_lo + o);
        const uint64_t dbh = smem_desc_sw128(b_hi + o), dbl = smem_desc_sw128(b_lo + o);
        mma_tf32(tmem, dal, dbh, idesc, (kt == 0 && ks == 0) ? 0u : 1u);
        mma_tf32(tmem, dah, dbl, idesc, 1u);
        mma_tf32(tmem, dah, dbh, idesc, 1u);
      }
      mma_commit(empty0 + 8 * s);
    }
    // arrives once every MMA issued above has completed
    mma_commit(done);
  }
  __syncwarp();
  if (nkt > 0 && !mbar_wait(done, 0, lim)) bs.timed_out = 1;
  tc_fence_after();
  __syncthreads();
  const bool ok = !bs.timed_out;  // the same for every thread after the barrier
  constexpr int ld = TN + 4;      // row pitch of the staged tile: 16-byte rows, no bank conflicts
  static_assert((size_t)TM * ld * 4 <= Sh::kRing, "staged tile must fit in the ring");
  if (ok) {
    // lane i of warp w holds row 32 w + i: two 16-byte stores per 8 columns
    const int i = warp * 32 + lane;
#pragma unroll 1
    for (int j0 = 0; j0 < TN; j0 += 8) {
      float v[8];
      if (nkt > 0) {
        tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0, v);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = 0.0f;
      }
      *reinterpret_cast<float4*>(smem + i * ld + j0) = make_float4(v[0], v[1], v[2], v[3]);
      *reinterpret_cast<float4*>(smem + i * ld + j0 + 4) = make_float4(v[4], v[5], v[6], v[7]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, Sh::kCols);
  if (ok) epi(static_cast<const float*>(smem), ld);
  return ok;
}

}  // namespace umma
}  // namespace cls
