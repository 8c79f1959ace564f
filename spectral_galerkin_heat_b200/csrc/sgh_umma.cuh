// sgh_umma.cuh -- split-BF16 contractions on the 5th-generation tensor cores
// (tcgen05.mma, accumulator in tensor memory), shared by the kernels that use
// them.
//
// * PTX wrappers: mbarriers with bounded waits, TMEM allocation, shared-memory
//   matrix descriptors (K-major, no swizzle, 8 x 8 core matrices of 128
//   contiguous bytes), the kind::f16 instruction descriptor, tcgen05.mma /
//   commit / ld, and bulk global -> shared copies completing on an mbarrier.
// * tile_bf16x3: one 128 x NT tile of D[m][n] = sum_k A(m, k) B(n, k) for FP64
//   operands delivered by loader functors. Each operand is split into BF16
//   hi + lo (x = hi + lo + O(2^-18 x)); per 16-wide k-step the tile issues
//   three MMAs -- hi*hi, hi*lo, lo*hi -- accumulating in FP32. The CTA's
//   threads stage the operands (converted on the way) double-buffered over
//   32-wide k-chunks; one thread issues the MMAs. Used by the stand-alone
//   tensor-core face DCT (sgh_mixed.cu).
// * Operand planes: BF16 hi / lo copies of an operand laid out chunk by chunk
//   exactly as a shared-memory stage, so that one bulk copy moves a chunk.
//   The batched fused face transform (sgh_batch.cu) streams its operands from
//   these planes.
//
// Every wait on an mbarrier is bounded: on expiry the caller records an error,
// waits (again bounded) for its work in flight, frees its tensor memory and
// returns without writing results.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sgh {
namespace umma {

constexpr int THREADS = 128;  // 4 warps; warp w owns accumulator lanes 32w..32w+31
constexpr int TM = 128;       // tile rows (UMMA M)
constexpr int KC = 32;        // k-chunk per stage (2 MMA k-steps)
constexpr unsigned WAIT_LIMIT = 1u << 22;  // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// true once the phase with the given parity has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  unsigned limit = WAIT_LIMIT) {
  for (unsigned i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}

// Warp-collective tensor-memory allocation; the column base lands in *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}

// Shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance
// between the two 8-element K halves of a 16-wide k-step, sbo = byte distance
// between consecutive 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of this architecture
  return d;                 // base offset 0, swizzle none
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (+)= A B^T, issued by one thread; no output lanes disabled.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t z = 0u;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
      smem_u32(bar)));
}

// 32 lanes x 16 consecutive 32-bit columns: this thread's lane, columns col..col+15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (r, k) of an R x KC K-major no-swizzle operand.
__device__ __forceinline__ uint32_t core_off(int r, int k, int R) {
  return (uint32_t)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn((float)x);
  lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

// Dynamic shared memory of one tile (bytes).
__host__ __device__ constexpr int smem_bytes(int NT) { return 2 * (2 * TM * KC * 2 + 2 * NT * KC * 2) + 64; }
// (layout: 2 stages of {A hi, A lo, B hi, B lo}, then 2 mbarriers, the TMEM
// address slot at +16 and the wait-outcome flag at +32)

// One 128 x NT tile (NT a multiple of 16 in [16, 256]). la(m, k) / lb(n, k)
// return the FP64 operand values (0 outside the problem); epi(m, n, value)
// receives each in-range result (m < M, n < N). Call from all 128 threads.
template <int NT, class LA, class LB, class EPI>
__device__ void tile_bf16x3(int M, int N, int K, int m0, int n0, const LA& la, const LB& lb, const EPI& epi,
                            char* smem, int* err) {
  constexpr int A_BYTES = TM * KC * 2;     // one split part of A per stage
  constexpr int B_BYTES = NT * KC * 2;
  constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
  constexpr uint32_t NCOLS = NT <= 32 ? 32 : (NT <= 64 ? 64 : (NT <= 128 ? 128 : 256));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * STAGE);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 2 * STAGE + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t idesc = idesc_bf16_f32(TM, NT);

  if (warp == 0) tmem_alloc(tslot, NCOLS);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  const int nchunks = (K + KC - 1) / KC;
  uint32_t phase[2] = {0u, 0u};
  // Only thread 0 waits on the barriers; the outcome is broadcast through
  // shared memory so every thread takes the same path.
  volatile int* okflag = reinterpret_cast<volatile int*>(smem + 2 * STAGE + 32);
  if (tid == 0) *okflag = 1;
  __syncthreads();
  bool ok = true;
  for (int ch = 0; ch < nchunks; ++ch) {
    const int b = ch & 1;
    if (ch >= 2) {  // buffer b was read by the MMAs of chunk ch-2
      if (tid == 0 && !mbar_wait_bounded(&bars[b], phase[b])) *okflag = 0;
      phase[b] ^= 1u;
      __syncthreads();
      if (!*okflag) {
        ok = false;
        break;
      }
    }
    char* st = smem + b * STAGE;
    const int k0 = ch * KC;
    for (int e = tid; e < TM * KC; e += THREADS) {  // A: k fastest across threads
      const int r = e / KC, k = e % KC;
      const int m = m0 + r, kk = k0 + k;
      const double x = (m < M && kk < K) ? la(m, kk) : 0.0;
      __nv_bfloat16 hi, lo;
      split_bf16(x, hi, lo);
      const uint32_t o = core_off(r, k, TM);
      *reinterpret_cast<__nv_bfloat16*>(st + o) = hi;
      *reinterpret_cast<__nv_bfloat16*>(st + A_BYTES + o) = lo;
    }
    for (int e = tid; e < NT * KC; e += THREADS) {
      const int r = e / KC, k = e % KC;
      const int n = n0 + r, kk = k0 + k;
      const double x = (n < N && kk < K) ? lb(n, kk) : 0.0;
      __nv_bfloat16 hi, lo;
      split_bf16(x, hi, lo);
      const uint32_t o = core_off(r, k, NT);
      *reinterpret_cast<__nv_bfloat16*>(st + 2 * A_BYTES + o) = hi;
      *reinterpret_cast<__nv_bfloat16*>(st + 2 * A_BYTES + B_BYTES + o) = lo;
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a_hi = smem_u32(st), a_lo = a_hi + A_BYTES;
      const uint32_t b_hi = a_hi + 2 * A_BYTES, b_lo = b_hi + B_BYTES;
#pragma unroll
      for (int s = 0; s < KC / 16; ++s) {
        const uint32_t ao = (uint32_t)(2 * s * (TM / 8) * 128), bo = (uint32_t)(2 * s * (NT / 8) * 128);
        const uint64_t dah = smem_desc(a_hi + ao, (TM / 8) * 128, 128);
        const uint64_t dal = smem_desc(a_lo + ao, (TM / 8) * 128, 128);
        const uint64_t dbh = smem_desc(b_hi + bo, (NT / 8) * 128, 128);
        const uint64_t dbl = smem_desc(b_lo + bo, (NT / 8) * 128, 128);
        const uint32_t acc0 = (ch > 0 || s > 0) ? 1u : 0u;
        mma_bf16(tmem, dah, dbh, idesc, acc0);
        mma_bf16(tmem, dah, dbl, idesc, 1u);
        mma_bf16(tmem, dal, dbh, idesc, 1u);
      }
      mma_commit(&bars[b]);
    }
  }
  // wait for the last commit (it covers every MMA issued before it)
  if (ok && nchunks > 0) {
    const int b = (nchunks - 1) & 1;
    if (tid == 0 && !mbar_wait_bounded(&bars[b], phase[b])) *okflag = 0;
    __syncthreads();
    ok = *okflag != 0;
  }
  if (!ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      // drain: give in-flight MMAs a bounded chance to finish before freeing TMEM
      for (int b = 0; b < 2; ++b) mbar_wait_bounded(&bars[b], phase[b]);
    }
  } else {
    tc_fence_after();
    const int m = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < NT; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      if (m < M) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (n0 + c + i < N) epi(m, n0 + c + i, (double)v[i]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
}

// ---------------------------------------------------------------------------
// Operand planes fed by bulk copies
// ---------------------------------------------------------------------------
// A plane holds one BF16 part (hi or lo) of an R x K operand, K-major, cut into
// 128-row x 32-wide chunks of 8 KB; each chunk is contiguous and laid out in
// core matrices exactly as the shared-memory stage (core_off), so one bulk
// copy moves it. Chunk (rt, kc) sits at byte (rt * nkc + kc) * CHUNK_BYTES.
// Rows and k beyond the operand are zero (planes are cleared once).
constexpr int CHUNK_BYTES = TM * KC * 2;  // 8192

__host__ __device__ inline size_t plane_bytes(int rows, int k) {
  return (size_t)((rows + TM - 1) / TM) * (size_t)((k + KC - 1) / KC) * CHUNK_BYTES;
}
__device__ __forceinline__ size_t plane_off(int r, int k, int nkc) {
  const int rt = r / TM, kc = k / KC;
  return (size_t)(rt * nkc + kc) * CHUNK_BYTES + core_off(r % TM, k % KC, TM);
}
__device__ __forceinline__ void plane_put(__nv_bfloat16* hi, __nv_bfloat16* lo, int r, int k, int nkc, double x) {
  __nv_bfloat16 h, l;
  split_bf16(x, h, l);
  const size_t o = plane_off(r, k, nkc) / 2;
  hi[o] = h;
  lo[o] = l;
}

// The same layout with R-row chunks (R = 64 or 128): chunk (r / R, k / KC)
// of R * KC * 2 bytes, core matrices as core_off(r % R, k % KC, R).
template <int R>
__host__ __device__ inline size_t plane_bytes_r(int rows, int k) {
  return (size_t)((rows + R - 1) / R) * (size_t)((k + KC - 1) / KC) * (size_t)(R * KC * 2);
}
template <int R>
__device__ __forceinline__ void plane_put_r(__nv_bfloat16* hi, __nv_bfloat16* lo, int r, int k, int nkc,
                                            double x) {
  __nv_bfloat16 h, l;
  split_bf16(x, h, l);
  const size_t o = ((size_t)((r / R) * nkc + k / KC) * (R * KC * 2) + core_off(r % R, k % KC, R)) / 2;
  hi[o] = h;
  lo[o] = l;
}

// Pair planes: the hi and lo parts of each chunk sit next to each other (hi at
// 2 ci C, lo at 2 ci C + C for chunk index ci = (r / R) nkc + k / KC and
// C = R * KC * 2 bytes), so ONE bulk copy moves both parts of a chunk. The
// shared-memory stage then holds hi followed by lo, as the MMAs read them.
template <int R>
__host__ __device__ constexpr size_t pair_chunk_bytes() { return (size_t)R * KC * 2; }
template <int R>
__host__ __device__ inline size_t pair_bytes(int rows, int k) { return 2 * plane_bytes_r<R>(rows, k); }
template <int R>
__device__ __forceinline__ size_t pair_off(int r, int k, int nkc) {
  return (size_t)((r / R) * nkc + k / KC) * 2 * pair_chunk_bytes<R>() + core_off(r % R, k % KC, R);
}
template <int R>
__device__ __forceinline__ void pair_put(char* plane, int r, int k, int nkc, double x) {
  __nv_bfloat16 h, l;
  split_bf16(x, h, l);
  const size_t o = pair_off<R>(r, k, nkc);
  *reinterpret_cast<__nv_bfloat16*>(plane + o) = h;
  *reinterpret_cast<__nv_bfloat16*>(plane + o + pair_chunk_bytes<R>()) = l;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace umma
}  // namespace sgh
