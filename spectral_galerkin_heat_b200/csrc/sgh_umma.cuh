// sgh_umma.cuh -- split-BF16 contraction tiles on the 5th-generation tensor
// cores (tcgen05.mma, accumulator in tensor memory).
//
// One CTA of 128 threads computes a 128 x NT tile of
//     D[m][n] = sum_k A(m, k) B(n, k)
// for FP64 operands A, B delivered by loader functors. Each operand is split
// into BF16 hi + lo parts (x = hi + lo + O(2^-16 x)); per 16-wide k-step the
// tile issues three kind::f16 MMAs -- hi*hi, hi*lo, lo*hi -- accumulating in
// FP32 in tensor memory. Operands are staged by the CTA's threads into shared
// memory (converted on the way, so no TMA), K-major, no swizzle, in 8 x 8
// "core matrices" of 128 contiguous bytes, double-buffered over 32-wide
// k-chunks; one elected thread issues the MMAs and commits them to an
// mbarrier per buffer.
//
// Every wait on an mbarrier is bounded: on expiry the tile records an error
// code in *err, waits (again bounded) for its MMAs, frees its tensor memory
// and returns without writing results.
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

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (unsigned i = 0; i < WAIT_LIMIT; ++i)
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

// 8 consecutive k (k0 % 8 == 0) of row r: one 16-byte row of a core matrix
// in each plane, written with one vector store per part.
__device__ __forceinline__ void plane_put8(__nv_bfloat16* hi, __nv_bfloat16* lo, int r, int k0, int nkc,
                                           const double (&x)[8]) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    __nv_bfloat16 h0, l0, h1, l1;
    split_bf16(x[2 * j], h0, l0);
    split_bf16(x[2 * j + 1], h1, l1);
    h[j] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
    l[j] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
  }
  const size_t o = plane_off(r, k0, nkc);
  *reinterpret_cast<uint4*>(reinterpret_cast<char*>(hi) + o) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(reinterpret_cast<char*>(lo) + o) = make_uint4(l[0], l[1], l[2], l[3]);
}

// ---- plane tiles: a ring of bulk-copy stages feeding the tensor cores -----
constexpr int PLANE_STAGES = 6;                 // k-chunks in flight
constexpr int PLANE_THREADS = 256;              // 2 warpgroups
constexpr int STAGE_BYTES = 4 * CHUNK_BYTES;    // A hi, A lo, B hi, B lo
// Dynamic shared memory of tile_planes (bytes): the stage ring, then barriers.
__host__ __device__ constexpr int planes_smem_bytes() { return PLANE_STAGES * STAGE_BYTES + 256; }

// FP32 result tile left in shared memory by tile_planes (it reuses the first
// 64 KB of the stage ring once every MMA has completed). Element (m, n) sits
// at float m * 128 + (n ^ (m & 31)): the XOR spreads a column over all 32
// banks for the TMEM -> shared copy and keeps rows conflict-free.
__device__ __forceinline__ float tile_value(const char* smem, int m, int n) {
  return reinterpret_cast<const float*>(smem)[m * 128 + (n ^ (m & 31))];
}

// One 128 x 128 tile D[m][n] = sum_k A(m, k) B(n, k) from operand planes.
// a_hi/a_lo point at chunk (rt, 0) of A's planes, b_hi/b_lo at chunk (ct, 0)
// of B's; nkc chunks along k. Thread 0 drives the ring: it issues the bulk
// copies of the first PLANE_STAGES chunks at once, then per chunk waits for
// its data, issues the three split-BF16 MMAs per 16-wide k-step, commits them,
// and refills the stage of the previous chunk as soon as that chunk's MMAs
// have drained. All waits are bounded: on expiry *err is set, in-flight work
// is waited for (bounded), tensor memory is freed and false is returned.
// On success the tile is in shared memory (tile_value) when this returns.
// Call from all PLANE_THREADS threads.
static __device__ bool tile_planes(const char* a_hi, const char* a_lo, const char* b_hi, const char* b_lo,
                                   int nkc, char* smem, int* err) {
  constexpr uint32_t NT = 128, NCOLS = 128;
  constexpr int S = PLANE_STAGES;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE_BYTES);
  uint64_t* done = full + S;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + S);
  volatile int* okflag = reinterpret_cast<volatile int*>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t idesc = idesc_bf16_f32(TM, NT);

  if (warp == 0) tmem_alloc(tslot, NCOLS);
  if (tid == 0) {
    for (int b = 0; b < S; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&done[b], 1);
    }
    *okflag = 1;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (tid == 0) {
    uint32_t fph = 0u, dph = 0u;  // parity bit per stage
    bool ok = true;
    auto load = [&](int ch) {
      const int b = ch % S;
      char* st = smem + b * STAGE_BYTES;
      const size_t off = (size_t)ch * CHUNK_BYTES;
      mbar_expect_tx(&full[b], STAGE_BYTES);
      bulk_g2s(st, a_hi + off, CHUNK_BYTES, &full[b]);
      bulk_g2s(st + CHUNK_BYTES, a_lo + off, CHUNK_BYTES, &full[b]);
      bulk_g2s(st + 2 * CHUNK_BYTES, b_hi + off, CHUNK_BYTES, &full[b]);
      bulk_g2s(st + 3 * CHUNK_BYTES, b_lo + off, CHUNK_BYTES, &full[b]);
    };
    const int pre = nkc < S ? nkc : S;
    for (int ch = 0; ch < pre; ++ch) load(ch);
    for (int ch = 0; ch < nkc; ++ch) {
      const int b = ch % S;
      if (!mbar_wait_bounded(&full[b], (fph >> b) & 1u)) { ok = false; break; }
      fph ^= 1u << b;
      tc_fence_after();
      const uint32_t s0 = smem_u32(smem + b * STAGE_BYTES);
      const uint32_t ah = s0, al = s0 + CHUNK_BYTES, bh = s0 + 2 * CHUNK_BYTES, bl = s0 + 3 * CHUNK_BYTES;
#pragma unroll
      for (int s = 0; s < KC / 16; ++s) {
        const uint32_t o = (uint32_t)(2 * s * (TM / 8) * 128);
        const uint64_t dah = smem_desc(ah + o, (TM / 8) * 128, 128);
        const uint64_t dal = smem_desc(al + o, (TM / 8) * 128, 128);
        const uint64_t dbh = smem_desc(bh + o, (TM / 8) * 128, 128);
        const uint64_t dbl = smem_desc(bl + o, (TM / 8) * 128, 128);
        mma_bf16(tmem, dah, dbh, idesc, (ch > 0 || s > 0) ? 1u : 0u);
        mma_bf16(tmem, dah, dbl, idesc, 1u);
        mma_bf16(tmem, dal, dbh, idesc, 1u);
      }
      mma_commit(&done[b]);
      // the stage of chunk ch-1 takes chunk ch-1+S once its MMAs are done
      if (ch >= 1 && ch - 1 + S < nkc) {
        const int pb = (ch - 1) % S;
        if (!mbar_wait_bounded(&done[pb], (dph >> pb) & 1u)) { ok = false; break; }
        dph ^= 1u << pb;
        load(ch - 1 + S);
      }
    }
    // the last commit covers every MMA issued before it
    if (ok && nkc > 0) {
      const int b = (nkc - 1) % S;
      if (!mbar_wait_bounded(&done[b], (dph >> b) & 1u)) ok = false;
    }
    if (!ok) {
      atomicExch(err, 1);
      *okflag = 0;
      for (int b = 0; b < S; ++b) {  // drain (bounded) before the memory is reused
        mbar_wait_bounded(&full[b], (fph >> b) & 1u);
        mbar_wait_bounded(&done[b], (dph >> b) & 1u);
      }
    }
  }
  __syncthreads();
  const bool good = *okflag != 0;
  if (good) {
    // warps w and w + 4 read TMEM lanes 32 (w % 4) .. +31, one column half each
    tc_fence_after();
    const int q = warp & 3, half = warp >> 2;
    const int m = q * 32 + lane;
    float* tile = reinterpret_cast<float*>(smem);
#pragma unroll 1
    for (int c = half * 64; c < half * 64 + 64; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) tile[m * 128 + ((c + i) ^ (m & 31))] = v[i];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
  return good;
}

}  // namespace umma
}  // namespace sgh
