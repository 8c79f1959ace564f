// sgh_axis.cuh -- one axis of a separable orthonormal DCT as a dense FP64
// contraction, with a fused per-element epilogue.
//
// View the C-ordered field as [A][N][B] with N the transformed axis. One pass
// computes out[a][k][b] = sum_n Mat[k][n] * in[a][n][b], i.e. the GEMM
// C[k, c] = sum_n Mat[k, n] X[n, c] with c = a*B + b. Mat is Nout x Nin: the
// orthonormal DCT-II matrix (forward), its transpose (DCT-III, inverse), or
// either with extra output rows appended (Nout > Nin) that yield face values
// from the same contraction (see the z-pass of the volume transforms). Three
// passes give scipy.fft.dctn(type=2|3, norm='ortho') over all axes
// (physics/spectral_cpu_kernels.py:374-389), two passes the face transform.
//
// Tiling: 256 threads; contraction slices stream through a 3-stage cp.async
// pipeline of 16-slice stages in shared memory; each thread owns a 2 x 4
// register tile (1 x 1 for passes too small to fill the SMs otherwise). When
// B == 1 (the transformed axis is the contiguous one) the fast dimension of
// the thread tile runs along k so that the epilogue stores are coalesced;
// when B > 1 it runs along c (= b, contiguous).
//
// The epilogue functor receives (linear output index (a*Nout + k)*B + b, k, b,
// value) and may accumulate two partial sums or a max that are reduced per CTA
// and written to a partials array (deterministic order).
#pragma once
#include <utility>

#include "sgh_device.cuh"
#include "sgh_umma.cuh"

namespace sgh {

constexpr int AX_THREADS = 256;
constexpr int AX_BK = 16;      // contraction slices per pipeline stage
constexpr int AX_STAGES = 3;   // cp.async pipeline depth

struct Red {
  double s0 = 0.0, s1 = 0.0, mx = -INFINITY;
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// 16 x 16 threads; each owns a TI (slow) x TJ (fast) register tile. The fast
// thread index runs along the contiguous output dimension: k when B == 1
// (CONTIG), c otherwise. Mat and X panels stream through an AX_STAGES-deep
// cp.async pipeline of AX_BK-slice stages (out-of-range elements zero-filled).
// Computes the output tile at (c0, k0) and hands every element to epi; the
// caller reduces r over the block.
template <bool CONTIG, int TI, int TJ, class Epi, class T = double>
__device__ __forceinline__ void axis_tile(const double* __restrict__ X, const double* __restrict__ Mat,
                                          int Nout, int N, int A, int B, int c0, int k0, const Epi& epi,
                                          Red& r) {
  // T: the arithmetic of the contraction -- double, or float for the FP32
  // plans (operands rounded to FP32 as they are read, FP32 products and sums)
  constexpr int TK = CONTIG ? 16 * TJ : 16 * TI;  // outputs along the transformed axis per tile
  constexpr int TC = CONTIG ? 16 * TI : 16 * TJ;  // outputs along c per tile
  __shared__ double Ms[AX_STAGES][AX_BK][TK + 1];
  __shared__ double Xs[AX_STAGES][AX_BK][TC + 1];

  const int tid = threadIdx.x;
  const int f = tid & 15;   // fast index
  const int s = tid >> 4;   // slow index
  const int ncol = A * B;
  const int nchunks = (N + AX_BK - 1) / AX_BK;

  auto issue = [&](int stage, int n0) {
    for (int e = tid; e < TK * AX_BK; e += AX_THREADS) {
      const int kr = e / AX_BK, kk = e % AX_BK;
      const int k = k0 + kr, n = n0 + kk;
      const bool ok = k < Nout && n < N;
      cp_async8(&Ms[stage][kk][kr], ok ? Mat + (size_t)k * N + n : Mat, ok ? 8 : 0);
    }
    if (CONTIG) {
      for (int e = tid; e < TC * AX_BK; e += AX_THREADS) {
        const int cr = e / AX_BK, kk = e % AX_BK;
        const int c = c0 + cr, n = n0 + kk;
        const bool ok = c < ncol && n < N;
        cp_async8(&Xs[stage][kk][cr], ok ? X + (size_t)c * N + n : X, ok ? 8 : 0);
      }
    } else {
      for (int e = tid; e < TC * AX_BK; e += AX_THREADS) {
        const int cr = e % TC, kk = e / TC;
        const int c = c0 + cr, n = n0 + kk;
        const bool ok = c < ncol && n < N;
        const double* src = X;
        if (ok) {
          const int a = c / B, b = c - a * B;
          src = X + ((size_t)a * N + n) * B + b;
        }
        cp_async8(&Xs[stage][kk][cr], src, ok ? 8 : 0);
      }
    }
    cp_async_commit();
  };

  T acc[TI][TJ];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int j = 0; j < TJ; ++j) acc[i][j] = T(0);

#pragma unroll
  for (int st = 0; st < AX_STAGES - 1; ++st) {
    if (st < nchunks) issue(st, st * AX_BK);
    else cp_async_commit();
  }
  for (int ch = 0; ch < nchunks; ++ch) {
    cp_async_wait<AX_STAGES - 2>();
    __syncthreads();
    const int nxt = ch + AX_STAGES - 1;
    if (nxt < nchunks) issue(nxt % AX_STAGES, nxt * AX_BK);
    else cp_async_commit();
    const int stg = ch % AX_STAGES;
#pragma unroll
    for (int kk = 0; kk < AX_BK; ++kk) {
      T m[CONTIG ? TJ : TI], x[CONTIG ? TI : TJ];
      if (CONTIG) {
#pragma unroll
        for (int j = 0; j < TJ; ++j) m[j] = (T)Ms[stg][kk][f + 16 * j];
#pragma unroll
        for (int i = 0; i < TI; ++i) x[i] = (T)Xs[stg][kk][TI * s + i];
#pragma unroll
        for (int i = 0; i < TI; ++i)
#pragma unroll
          for (int j = 0; j < TJ; ++j) acc[i][j] = fma(m[j], x[i], acc[i][j]);
      } else {
#pragma unroll
        for (int i = 0; i < TI; ++i) m[i] = (T)Ms[stg][kk][TI * s + i];
#pragma unroll
        for (int j = 0; j < TJ; ++j) x[j] = (T)Xs[stg][kk][f + 16 * j];
#pragma unroll
        for (int i = 0; i < TI; ++i)
#pragma unroll
          for (int j = 0; j < TJ; ++j) acc[i][j] = fma(m[i], x[j], acc[i][j]);
      }
    }
  }
  cp_async_wait<0>();

#pragma unroll
  for (int i = 0; i < TI; ++i) {
#pragma unroll
    for (int j = 0; j < TJ; ++j) {
      const int k = CONTIG ? (k0 + f + 16 * j) : (k0 + TI * s + i);
      const int c = CONTIG ? (c0 + TI * s + i) : (c0 + f + 16 * j);
      if (k < Nout && c < ncol) {
        const int a = c / B, b = c - a * B;
        const int idx = (a * Nout + k) * B + b;
        epi(idx, k, b, (double)acc[i][j], r);
      }
    }
  }
}

template <bool CONTIG, int TI, int TJ, class Epi, class T = double>
__global__ void __launch_bounds__(AX_THREADS)
k_axis(const double* __restrict__ X, const double* __restrict__ Mat, int Nout, int N, int A, int B,
       Epi epi) {
  constexpr int TK = CONTIG ? 16 * TJ : 16 * TI;
  constexpr int TC = CONTIG ? 16 * TI : 16 * TJ;
  __shared__ double red_sh[2 * (AX_THREADS / 32)];
  // programmatic stream serialisation: nothing global before the previous kernel completes
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  Red r;
  axis_tile<CONTIG, TI, TJ, Epi, T>(X, Mat, Nout, N, A, B, blockIdx.x * TC, blockIdx.y * TK, epi, r);
  if (Epi::kReduce) {
    double p0, p1;
    if (Epi::kReduce == 1) {
      p0 = r.s0;
      p1 = r.s1;
      block_sum2<AX_THREADS>(p0, p1, red_sh);
    } else {
      p0 = r.mx;
      p1 = r.s0;
      block_max_sum<AX_THREADS>(p0, p1, red_sh);
    }
    if (threadIdx.x == 0) {
      const int blk = blockIdx.y * gridDim.x + blockIdx.x;
      epi.partials[2 * blk] = p0;
      epi.partials[2 * blk + 1] = p1;
    }
  }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core variant: mma.sync m16n8k8 .f64 (the FP64 MMA of sm_90+,
// kept on sm_100a; tcgen05 has no FP64 kind). CTA tile BM (outputs along the
// transformed axis) x BN (columns c), 8 warps as 2 x 4, warp tile BM/2 x BN/4
// = BM/32 m16 x BN/32 n8 MMA tiles per k8 step. Mat and X tiles stream through an
// cp.async pipeline of AXM_BK-slice stages, as deep as about 96 KB of shared
// memory allows (3 to 6 stages: small tiles compute little per stage, so
// more stages stay in flight to cover the L2 latency). Shared layouts keep the
// fragment reads and the cp.async writes free of bank conflicts: Mat tiles
// k-major rows of AXM_BK + 4 doubles; X tiles column-major (rows of AXM_BK + 4)
// when the contraction axis is the contiguous one (B == 1), else n-major rows
// of BN + 4. Each thread's source columns are fixed across stages, so their
// offsets are computed once.
// ---------------------------------------------------------------------------
constexpr int AXM_BK = 16;
constexpr int AXM_SMEM_TARGET = 96 * 1024;
constexpr int AXM_LDK = AXM_BK + 4;  // rows of AXM_BK contraction slices

template <bool CONTIG, int BM, int BN>
constexpr int axm_stage_doubles() {
  return BM * AXM_LDK + (CONTIG ? BN * AXM_LDK : AXM_BK * (BN + 4));
}
template <bool CONTIG, int BM, int BN>
constexpr int axm_stages() {
  constexpr int n = AXM_SMEM_TARGET / (axm_stage_doubles<CONTIG, BM, BN>() * (int)sizeof(double));
  return n < 3 ? 3 : (n > 6 ? 6 : n);
}
template <bool CONTIG, int BM, int BN>
constexpr int axm_smem_bytes() {
  return axm_stages<CONTIG, BM, BN>() * axm_stage_doubles<CONTIG, BM, BN>() * (int)sizeof(double);
}

__device__ __forceinline__ void mma_f64_m16n8k8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <bool CONTIG, int BM, int BN, class Epi>
__global__ void __launch_bounds__(AX_THREADS)
k_axis_mma(const double* __restrict__ X, const double* __restrict__ Mat, int Nout, int N, int A, int B,
           Epi epi) {
  static_assert(BM == 32 || BM == 64, "BM");
  static_assert(BN == 64 || BN == 128, "BN");
  extern __shared__ __align__(16) double axm_sh[];
  constexpr int STAGE = axm_stage_doubles<CONTIG, BM, BN>();
  constexpr int LDX = CONTIG ? AXM_LDK : BN + 4;
  constexpr int MT = BM / 32;           // m16 tiles per warp (warp rows BM / 2)
  constexpr int NT = BN / 32;           // n8 tiles per warp
  constexpr int XPT = BN * AXM_BK / AX_THREADS;  // X elements per thread per stage
  __shared__ double red_sh[2 * (AX_THREADS / 32)];

  // Launched with programmatic stream serialisation: wait for the previous
  // kernel of the stream (complete, memory visible) before the first global
  // access of any kind, so neither its outputs nor the buffers it still reads
  // are touched early. Only the launch and this prologue overlap its tail.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;
  const int ncol = A * B;
  const int c0 = blockIdx.x * BN, k0 = blockIdx.y * BM;
  const int nchunks = (N + AXM_BK - 1) / AXM_BK;

  // 16-byte copies of element pairs where every pair is aligned and lies
  // wholly inside or outside the array: along n for Mat (and X when B == 1)
  // when N is even, along c for X when B is even. Uniform per launch.
  const bool vecM = (N % 2 == 0) && (reinterpret_cast<uintptr_t>(Mat) % 16 == 0);
  const bool vecX = (CONTIG ? (N % 2 == 0) : (B % 2 == 0)) && (reinterpret_cast<uintptr_t>(X) % 16 == 0);

  // Mat tile: BM rows x AXM_BK slices, slices fastest. Scalar: BM / 16 per
  // thread, rows m_r0 + 16 j, slice m_kk. Pairs: BM / 32 per thread, rows
  // mp_r0 + 32 j, slices 2 mp_p, 2 mp_p + 1.
  const int m_kk = tid & 15, m_r0 = tid >> 4;
  const int mp_p = tid & 7, mp_r0 = tid >> 3;
  // X tile: per-thread column bases (fixed over the stages)
  int x_kk0, x_cr0;
  size_t xbase[CONTIG ? XPT : 1];
  bool xok[CONTIG ? XPT : 1];
  // pairs: CONTIG: pair xp_p (slices 2 xp_p, +1) of columns xp_c0 + 32 j;
  // otherwise columns 2 xp_c, 2 xp_c + 1 of slices xp_k0 + (2 AX_THREADS / BN) j
  const int xp_p = tid & 7, xp_c0 = tid >> 3;
  const int xp_c = tid % (BN / 2), xp_k0 = tid / (BN / 2);
  size_t xpbase = 0;
  bool xpok = false;
  if (CONTIG) {
    x_kk0 = tid & 15;
    x_cr0 = tid >> 4;  // columns x_cr0 + 16 j
#pragma unroll
    for (int j = 0; j < XPT; ++j) {
      const int c = c0 + x_cr0 + 16 * j;
      xok[j] = c < ncol;
      xbase[j] = (size_t)(xok[j] ? c : 0) * N;
    }
  } else {
    x_cr0 = tid % BN;
    x_kk0 = tid / BN;  // slices x_kk0 + (AX_THREADS / BN) j
    const int c = c0 + x_cr0;
    xok[0] = c < ncol;
    const int cc = xok[0] ? c : 0;
    const int a = cc / B, b = cc - a * B;
    xbase[0] = (size_t)a * N * B + b;
    // pair base: column c0 + 2 xp_c (even, so b is even when B is even)
    const int cp = c0 + 2 * xp_c;
    xpok = cp < ncol;
    const int cq = xpok ? cp : 0;
    const int ap = cq / B, bp = cq - ap * B;
    xpbase = (size_t)ap * N * B + bp;
  }

  auto issue = [&](int stage, int n0) {
    double* Ms = axm_sh + stage * STAGE;
    double* Xs = Ms + BM * AXM_LDK;
    if (vecM) {
      const int n = n0 + 2 * mp_p;
#pragma unroll
      for (int j = 0; j < BM / 32; ++j) {
        const int k = k0 + mp_r0 + 32 * j;
        const bool ok = k < Nout && n < N;
        cp_async16(&Ms[(mp_r0 + 32 * j) * AXM_LDK + 2 * mp_p], ok ? Mat + (size_t)k * N + n : Mat, ok ? 16 : 0);
      }
    } else {
      const int n = n0 + m_kk;
#pragma unroll
      for (int j = 0; j < BM / 16; ++j) {
        const int k = k0 + m_r0 + 16 * j;
        const bool ok = k < Nout && n < N;
        cp_async8(&Ms[(m_r0 + 16 * j) * AXM_LDK + m_kk], ok ? Mat + (size_t)k * N + n : Mat, ok ? 8 : 0);
      }
    }
    if (CONTIG) {
      if (vecX) {
        const int n = n0 + 2 * xp_p;
#pragma unroll
        for (int j = 0; j < XPT / 2; ++j) {
          const int cr = xp_c0 + 32 * j;
          const int c = c0 + cr;
          const bool ok = c < ncol && n < N;
          cp_async16(&Xs[cr * LDX + 2 * xp_p], ok ? X + (size_t)c * N + n : X, ok ? 16 : 0);
        }
      } else {
        const int n = n0 + x_kk0;
#pragma unroll
        for (int j = 0; j < XPT; ++j) {
          const bool ok = xok[j] && n < N;
          cp_async8(&Xs[(x_cr0 + 16 * j) * LDX + x_kk0], ok ? X + xbase[j] + n : X, ok ? 8 : 0);
        }
      }
    } else {
      if (vecX) {
        constexpr int KSTEP2 = 2 * AX_THREADS / BN;
#pragma unroll
        for (int j = 0; j < XPT / 2; ++j) {
          const int kk = xp_k0 + KSTEP2 * j;
          const int n = n0 + kk;
          const bool ok = xpok && n < N;
          cp_async16(&Xs[kk * LDX + 2 * xp_c], ok ? X + xpbase + (size_t)n * B : X, ok ? 16 : 0);
        }
      } else {
        constexpr int KSTEP = AX_THREADS / BN;
#pragma unroll
        for (int j = 0; j < XPT; ++j) {
          const int kk = x_kk0 + KSTEP * j;
          const int n = n0 + kk;
          const bool ok = xok[0] && n < N;
          cp_async8(&Xs[kk * LDX + x_cr0], ok ? X + xbase[0] + (size_t)n * B : X, ok ? 8 : 0);
        }
      }
    }
    cp_async_commit();
  };

  double acc[MT][NT][4];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

#pragma unroll
  constexpr int STAGES = axm_stages<CONTIG, BM, BN>();
  for (int st = 0; st < STAGES - 1; ++st) {
    if (st < nchunks) issue(st, st * AXM_BK);
    else cp_async_commit();
  }
  for (int ch = 0; ch < nchunks; ++ch) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int nxt = ch + STAGES - 1;
    if (nxt < nchunks) issue(nxt % STAGES, nxt * AXM_BK);
    else cp_async_commit();
    const double* Ms = axm_sh + (ch % STAGES) * STAGE;
    const double* Xs = Ms + BM * AXM_LDK;
#pragma unroll
    for (int k8 = 0; k8 < AXM_BK; k8 += 8) {
      // A fragment (row-major 16 x 8): a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4)
      double af[MT][4];
#pragma unroll
      for (int i = 0; i < MT; ++i) {
        const double* r0 = Ms + (wm * (BM / 2) + i * 16 + g) * AXM_LDK + k8 + t;
        const double* r1 = r0 + 8 * AXM_LDK;
        af[i][0] = r0[0];
        af[i][1] = r1[0];
        af[i][2] = r0[4];
        af[i][3] = r1[4];
      }
      // B fragment (col-major 8 x 8): b0 (k = t, n = g), b1 (k = t + 4, n = g)
      double bf[NT][2];
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int col = wn * (BN / 4) + j * 8 + g;
        if (CONTIG) {
          bf[j][0] = Xs[col * LDX + k8 + t];
          bf[j][1] = Xs[col * LDX + k8 + t + 4];
        } else {
          bf[j][0] = Xs[(k8 + t) * LDX + col];
          bf[j][1] = Xs[(k8 + t + 4) * LDX + col];
        }
      }
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) mma_f64_m16n8k8(acc[i][j], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();

  // Epilogue through shared memory: the D fragments (16 x 8: d0, d1 at
  // (g, 2t + {0, 1}), d2, d3 at (g + 8, 2t + {0, 1})) go to a BM x BN tile,
  // then every thread hands consecutive outputs to epi, contiguous in memory
  // (along k when B == 1, along c otherwise). Column offsets are computed
  // once per column.
  constexpr int LDT = BN + 1;
  double* tile = axm_sh;                                  // BM x LDT (fits in the stages)
  int* colbase = reinterpret_cast<int*>(tile + BM * LDT);      // BN: a * Nout * B + b
  int* colb = colbase + BN;                                    // BN: b
  static_assert((BM * (BN + 1)) * 8 + 2 * BN * 4 <= axm_smem_bytes<CONTIG, BM, BN>(), "epilogue tile");
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = wm * (BM / 2) + i * 16 + g + 8 * (q >> 1);
        const int col = wn * (BN / 4) + j * 8 + 2 * t + (q & 1);
        tile[row * LDT + col] = acc[i][j][q];
      }
  if (tid < BN) {
    const int c = c0 + tid;
    const int cc = c < ncol ? c : 0;
    const int a = cc / B, b = cc - a * B;
    colbase[tid] = a * Nout * B + b;
    colb[tid] = b;
  }
  __syncthreads();
  Red r;
  const int kmax = min(BM, Nout - k0), cmax = min(BN, ncol - c0);
  if (CONTIG) {
    for (int e = tid; e < BM * BN; e += AX_THREADS) {
      const int kr = e % BM, cr = e / BM;
      if (kr < kmax && cr < cmax) {
        const int k = k0 + kr;
        epi(colbase[cr] + k, k, 0, tile[kr * LDT + cr], r);
      }
    }
  } else {
    for (int e = tid; e < BM * BN; e += AX_THREADS) {
      const int cr = e % BN, kr = e / BN;
      if (kr < kmax && cr < cmax) {
        const int k = k0 + kr;
        epi(colbase[cr] + k * B, k, colb[cr], tile[kr * LDT + cr], r);
      }
    }
  }
  if (Epi::kReduce) {
    double p0, p1;
    if (Epi::kReduce == 1) {
      p0 = r.s0;
      p1 = r.s1;
      block_sum2<AX_THREADS>(p0, p1, red_sh);
    } else {
      p0 = r.mx;
      p1 = r.s0;
      block_max_sum<AX_THREADS>(p0, p1, red_sh);
    }
    if (threadIdx.x == 0) {
      const int blk = blockIdx.y * gridDim.x + blockIdx.x;
      epi.partials[2 * blk] = p0;
      epi.partials[2 * blk + 1] = p1;
    }
  }
}

// Launch with programmatic stream serialisation: the kernel may be scheduled
// while the previous kernel of the stream finishes, and must execute
// griddepcontrol.wait before its first global access (every kernel launched
// here does, in all CTAs).
template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, int threads, int smem, cudaStream_t st,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute la[1];
  la[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  la[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = la;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// ---------------------------------------------------------------------------
// Split-BF16 tensor-core variant (tcgen05, the mixed-precision plans). One CTA
// of 128 threads computes D[k][c] = sum_n Mat[k][n] X(c, n) for 128 outputs k
// of the transformed axis (the MMA's M; TMEM lane = output) and NC columns c
// (the MMA's N; TMEM column = column), so every column is read once per
// 128 outputs. The matrix operand arrives split into BF16 hi + lo: from the
// plan's pair plane of that matrix (one 16 KB bulk copy per 32-slice chunk,
// completing on the stage's mbarrier), or, for a matrix without a plane,
// split by the threads. The column operand is copied raw (FP64) by cp.async
// into a ring of S stages -- every thread copies and later splits the same
// elements -- and split into the MMA stage of the same index. Per 16-slice
// step one thread issues hi.hi, hi.lo, lo.hi, accumulating in FP32 in tensor
// memory. Contiguous passes (B == 1) hand each thread's output row to the
// epilogue straight from tensor memory (lanes = consecutive outputs of one
// column, so stores coalesce); strided passes transpose through shared memory
// so that consecutive threads take consecutive columns. Every mbarrier wait
// is bounded: on expiry the CTA sets *err, waits (bounded) for its bulk
// copies and MMAs in flight, writes NaN partials so the Picard test stops,
// frees its tensor memory and returns without results.
// ---------------------------------------------------------------------------
constexpr int AXU_THREADS = 128;
constexpr int AXU_M = 128;                            // outputs per CTA
constexpr int AXU_KC = 32;                            // contraction slices per stage
constexpr int AXU_ABYTES = 2 * AXU_M * AXU_KC * 2;    // matrix hi + lo of one stage (16 KB)
// Whether passes run on the split-BF16 tensor-core kernel (mixed-precision
// plans), and where that kernel records an expired wait.
inline thread_local bool g_axis_umma = false;
inline thread_local int* g_umma_err = nullptr;
// Whether passes run the CUDA-core kernel in FP32 arithmetic (FP32 plans).
inline thread_local bool g_axis_fp32 = false;

// A matrix of a plan with its BF16 pair plane (umma::pair_off<128> layout,
// rows and slices beyond the matrix zero): passes whose Mat is listed here
// with the same contraction length and no more outputs than rows stream
// the matrix operand from the plane.
struct UmmaPlane {
  const double* mat;
  const char* pair;
  int rows, k;
};
inline thread_local const UmmaPlane* g_umma_planes = nullptr;
inline thread_local int g_umma_nplanes = 0;
inline const char* umma_plane_for(const double* Mat, int Nout, int N) {
  for (int i = 0; i < g_umma_nplanes; ++i) {
    const UmmaPlane& q = g_umma_planes[i];
    if (q.mat == Mat && q.k == N && Nout <= q.rows) return q.pair;
  }
  return nullptr;
}

template <int NC>
__host__ __device__ constexpr int axu_stages() { return NC >= 64 ? 3 : 4; }
template <int NC>
__host__ __device__ constexpr int axu_bbytes() { return 2 * NC * AXU_KC * 2; }  // column operand hi + lo
template <int NC>
__host__ __device__ constexpr int axu_rbytes() { return NC * AXU_KC * 8; }      // raw FP64 columns
template <int NC>
__host__ __device__ constexpr int axu_stage_bytes() { return AXU_ABYTES + axu_bbytes<NC>() + axu_rbytes<NC>(); }
template <int NC>
__host__ __device__ constexpr int axu_smem_bytes() { return axu_stages<NC>() * axu_stage_bytes<NC>() + 128; }
// Column tile NC of a pass: the widest of 64, 32, 16 that still gives one
// wave of CTAs (one per SM), else 16.
inline int axu_nc(int Nout, int ncol) {
  constexpr long kSms = 148;
  const long mt = (Nout + AXU_M - 1) / AXU_M;
  int nc = 64;
  while (nc > 16 && mt * ((ncol + nc - 1) / nc) < kSms) nc /= 2;
  return nc;
}

// Builds the pair plane of an rows x k matrix (row-major, Mat[r * k + n]).
static __global__ void k_pair_plane(const double* __restrict__ M, int rows, int k, char* __restrict__ pair) {
  const int nkc = (k + AXU_KC - 1) / AXU_KC, kpad = nkc * AXU_KC;
  const long n = (long)((rows + AXU_M - 1) / AXU_M) * AXU_M * kpad;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const int r = (int)(e / kpad), kk = (int)(e % kpad);
    const double x = (r < rows && kk < k) ? M[(size_t)r * k + kk] : 0.0;
    umma::pair_put<AXU_M>(pair, r, kk, nkc, x);
  }
}

template <bool CONTIG, int NC, class Epi>
__global__ void __launch_bounds__(AXU_THREADS)
k_axis_umma(const double* __restrict__ X, const double* __restrict__ Mat, const char* __restrict__ pair,
            int Nout, int N, int A, int B, Epi epi, int* err) {
  using namespace umma;
  extern __shared__ __align__(128) char axu_sh[];
  __shared__ double red_sh[2 * (AXU_THREADS / 32)];
  constexpr int S = axu_stages<NC>(), BH = NC * AXU_KC * 2, STAGE = axu_stage_bytes<NC>();
  constexpr int PER = NC * AXU_KC / AXU_THREADS;  // column values per thread and chunk: 4 .. 16
  constexpr uint32_t NCOLS = NC < 32 ? 32 : NC;
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ncol = A * B;
  const int c0 = blockIdx.x * NC, k0 = blockIdx.y * AXU_M;
  uint64_t* full = reinterpret_cast<uint64_t*>(axu_sh + S * STAGE);
  uint64_t* empty = full + S;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(axu_sh + S * STAGE + 64);
  volatile int* okflag = reinterpret_cast<volatile int*>(axu_sh + S * STAGE + 72);
  const uint32_t idesc = idesc_bf16_f32(AXU_M, NC);
  const int nchunks = (N + AXU_KC - 1) / AXU_KC;
  const bool planed = pair != nullptr;
  if (warp == 0) tmem_alloc(tslot, NCOLS);
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    *okflag = 1;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  // element e = tid + i * 128 of a chunk: column j, slice nl; the raw ring
  // holds it at 8 e (contiguous passes: [column][slice], a warp copies 32
  // consecutive slices of a column; strided: [slice][column], consecutive
  // threads copy consecutive columns)
  auto elem = [&](int e, int& j, int& nl) {
    if (CONTIG) {
      j = e / AXU_KC;
      nl = e % AXU_KC;
    } else {
      nl = e / NC;
      j = e % NC;
    }
  };
  auto issue_raw = [&](int ch) {  // one commit group per chunk (empty past the end)
    if (ch < nchunks) {
      char* raw = axu_sh + (ch % S) * STAGE + AXU_ABYTES + 2 * BH;
      const int n0 = ch * AXU_KC;
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        const int e = tid + i * AXU_THREADS;
        int j, nl;
        elem(e, j, nl);
        const int c = c0 + j, n = n0 + nl;
        const bool in = c < ncol && n < N;
        size_t off = 0;
        if (in) {
          if (CONTIG) {
            off = (size_t)c * N + n;
          } else {
            const int a = c / B, b = c - a * B;
            off = (size_t)a * N * B + (size_t)n * B + b;
          }
        }
        cp_async8(raw + 8 * e, X + off, in ? 8 : 0);
      }
    }
    cp_async_commit();
  };
  auto issue_a = [&](int ch) {  // thread 0: the matrix chunk ch from the plane
    const int s = ch % S;
    mbar_expect_tx(&full[s], AXU_ABYTES);
    bulk_g2s(axu_sh + s * STAGE, pair + ((size_t)blockIdx.y * nchunks + ch) * AXU_ABYTES, AXU_ABYTES, &full[s]);
  };

  // thread 0's bookkeeping: matrix chunks copied (a_next) and consumed
  // (a_done), and the last chunk whose MMAs were committed
  int a_next = 0, a_done = 0, last_commit = -1;
  for (int ch = 0; ch < S; ++ch) issue_raw(ch);
  if (planed && tid == 0)
    for (; a_next < S && a_next < nchunks; ++a_next) issue_a(a_next);
  bool ok = true;
  for (int ch = 0; ch < nchunks; ++ch) {
    const int s = ch % S;
    char* st = axu_sh + s * STAGE;
    cp_async_wait<S - 1>();  // this thread's copies of chunk ch have landed
    __syncthreads();         // thread 0 saw the MMAs of chunk ch - S complete
    if (!*okflag) {
      ok = false;
      break;
    }
    const int n0 = ch * AXU_KC;
    if (!planed) {  // matrix rows k0.. of slices n0..: 32 values per thread
#pragma unroll 8
      for (int i = 0; i < AXU_M * AXU_KC / AXU_THREADS; ++i) {
        const int e = tid + i * AXU_THREADS, r = e / AXU_KC, kl = e % AXU_KC;
        const int k = k0 + r, n = n0 + kl;
        const double x = (k < Nout && n < N) ? __ldg(Mat + (size_t)k * N + n) : 0.0;
        __nv_bfloat16 h, l;
        split_bf16(x, h, l);
        const uint32_t o = core_off(r, kl, AXU_M);
        *reinterpret_cast<__nv_bfloat16*>(st + o) = h;
        *reinterpret_cast<__nv_bfloat16*>(st + AXU_ABYTES / 2 + o) = l;
      }
    }
    {
      const double* raw = reinterpret_cast<const double*>(st + AXU_ABYTES + 2 * BH);
      double xv[PER];
#pragma unroll
      for (int i = 0; i < PER; ++i) xv[i] = raw[tid + i * AXU_THREADS];
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        int j, nl;
        elem(tid + i * AXU_THREADS, j, nl);
        __nv_bfloat16 h, l;
        split_bf16(xv[i], h, l);
        const uint32_t o = core_off(j, nl, NC);
        *reinterpret_cast<__nv_bfloat16*>(st + AXU_ABYTES + o) = h;
        *reinterpret_cast<__nv_bfloat16*>(st + AXU_ABYTES + BH + o) = l;
      }
    }
    issue_raw(ch + S);  // into the slot this thread just read
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      bool good = true;
      if (planed) {
        good = mbar_wait_bounded(&full[s], (uint32_t)((ch / S) & 1));
        if (good) a_done = ch + 1;
      }
      if (good) {
        tc_fence_after();
        const uint32_t ah = smem_u32(st), al = ah + AXU_ABYTES / 2, bh = ah + AXU_ABYTES, bl = bh + BH;
#pragma unroll
        for (int q = 0; q < AXU_KC / 16; ++q) {
          const uint32_t ao = (uint32_t)(2 * q * (AXU_M / 8) * 128), bo = (uint32_t)(2 * q * (NC / 8) * 128);
          const uint64_t dah = smem_desc(ah + ao, (AXU_M / 8) * 128, 128);
          const uint64_t dal = smem_desc(al + ao, (AXU_M / 8) * 128, 128);
          const uint64_t dbh = smem_desc(bh + bo, (NC / 8) * 128, 128);
          const uint64_t dbl = smem_desc(bl + bo, (NC / 8) * 128, 128);
          const uint32_t acc = (ch > 0 || q > 0) ? 1u : 0u;
          mma_bf16(tmem, dah, dbh, idesc, acc);
          mma_bf16(tmem, dah, dbl, idesc, 1u);
          mma_bf16(tmem, dal, dbh, idesc, 1u);
        }
        mma_commit(&empty[s]);
        last_commit = ch;
        // stage (ch - 1) % S is reused by chunk ch - 1 + S: wait for the MMAs
        // of chunk ch - 1 (issued an iteration ago), then refill its matrix
        const int prev = ch - 1, next = ch - 1 + S;
        if (prev >= 0 && next < nchunks) {
          good = mbar_wait_bounded(&empty[prev % S], (uint32_t)((prev / S) & 1));
          if (good && planed) issue_a(a_next++);
        }
      }
      if (!good) *okflag = 0;
    }
  }
  cp_async_wait<0>();
  if (ok && nchunks > 0) {  // the last commit covers every MMA before it
    if (tid == 0 && !mbar_wait_bounded(&empty[(nchunks - 1) % S], (uint32_t)(((nchunks - 1) / S) & 1)))
      *okflag = 0;
    __syncthreads();
    ok = *okflag != 0;
  }
  Red r;
  if (!ok) {
    if (tid == 0) {
      if (err) atomicExch(err, 1);
      for (int c = a_done; c < a_next; ++c) mbar_wait_bounded(&full[c % S], (uint32_t)((c / S) & 1));
      if (last_commit >= 0) mbar_wait_bounded(&empty[last_commit % S], (uint32_t)((last_commit / S) & 1));
    }
  } else {
    tc_fence_after();
    fence_proxy_async();
    const int kl = warp * 32 + lane, k = k0 + kl;
    const bool live = k0 + warp * 32 < Nout;  // warp-uniform
    if (CONTIG) {
      if (live) {
#pragma unroll 1
        for (int j0 = 0; j0 < NC; j0 += 16) {
          float v[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0, v);
          if (k < Nout) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int c = c0 + j0 + i;
              if (c < ncol) epi(c * Nout + k, k, 0, (double)v[i], r);
            }
          }
        }
      }
    } else {
      float* T = reinterpret_cast<float*>(axu_sh);  // [128 outputs][NC + 1]
      if (live) {
#pragma unroll 1
        for (int j0 = 0; j0 < NC; j0 += 16) {
          float v[16];
          tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j0, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) T[kl * (NC + 1) + j0 + i] = v[i];
        }
      }
      __syncthreads();
      const int rows = min(AXU_M, Nout - k0);
      for (int e = tid; e < rows * NC; e += AXU_THREADS) {
        const int kk = e / NC, j = e - kk * NC, c = c0 + j;
        if (c < ncol) {
          const int a = c / B, b = c - a * B, kq = k0 + kk;
          epi(a * Nout * B + kq * B + b, kq, b, (double)T[kk * (NC + 1) + j], r);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, NCOLS);
  if (Epi::kReduce) {
    double p0, p1;
    if (Epi::kReduce == 1) {
      p0 = r.s0;
      p1 = r.s1;
      block_sum2<AXU_THREADS>(p0, p1, red_sh);
    } else {
      p0 = r.mx;
      p1 = r.s0;
      block_max_sum<AXU_THREADS>(p0, p1, red_sh);
    }
    if (threadIdx.x == 0) {
      const int blk = blockIdx.y * gridDim.x + blockIdx.x;
      epi.partials[2 * blk] = ok ? p0 : nan("");
      epi.partials[2 * blk + 1] = ok ? p1 : nan("");
    }
  }
}

template <bool CONTIG, int NC, class Epi>
inline void launch_axis_umma_nc(const double* X, const double* Mat, const char* pair, int Nout, int N, int A,
                                int B, const Epi& epi, dim3 grid, cudaStream_t st) {
  constexpr int bytes = axu_smem_bytes<NC>();
  static const bool attr = [] {
    cudaFuncSetAttribute(k_axis_umma<CONTIG, NC, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return true;
  }();
  (void)attr;
  launch_pdl(k_axis_umma<CONTIG, NC, Epi>, grid, AXU_THREADS, bytes, st, X, Mat, pair, Nout, N, A, B, epi,
             g_umma_err);
}

template <bool CONTIG, class Epi>
inline void launch_axis_umma(const double* X, const double* Mat, int Nout, int N, int A, int B, const Epi& epi,
                             dim3 grid, cudaStream_t st) {
  const char* pair = umma_plane_for(Mat, Nout, N);
  switch (axu_nc(Nout, A * B)) {
    case 16: launch_axis_umma_nc<CONTIG, 16>(X, Mat, pair, Nout, N, A, B, epi, grid, st); break;
    case 32: launch_axis_umma_nc<CONTIG, 32>(X, Mat, pair, Nout, N, A, B, epi, grid, st); break;
    default: launch_axis_umma_nc<CONTIG, 64>(X, Mat, pair, Nout, N, A, B, epi, grid, st); break;
  }
}

// Launch shape of one pass. kind 2..5: the FP64 tensor-core kernel with a
// BM x BN tile of 64 x 128, 64 x 64, 32 x 128, 32 x 64, when the pass is large
// enough (see axis_shape); kind 1: the 2 x 4 thread tile when it yields
// enough CTAs to cover the SMs; kind 0: the 1 x 1 tile (small faces, short axes).
struct AxisShape {
  bool big;
  dim3 grid;
  int kind = 0;
};
constexpr int AX_MIN_CTAS = 132;
// Tile policy of the calling thread: 2 x 4 tiles when that grid has at least
// this many CTAs. Set for the duration of a plan's call by AxisPolicy, so the
// captured graph, eager launches and the partial-buffer sizing agree.
inline thread_local int g_axis_min_ctas = AX_MIN_CTAS;
// Whether passes may use the FP64 tensor-core kernel (on by default; the
// CUDA-core kernels remain for small passes and for comparison).
inline thread_local bool g_axis_mma = true;
constexpr int AXM_SMS = 148;          // CTAs of one full wave at one CTA per SM
constexpr int AXM_MIN_CTAS = 16;      // smaller passes stay on the CUDA-core kernels

struct AxisPolicy {
  int saved;
  bool saved_mma, saved_umma, saved_fp32;
  int* saved_err;
  const UmmaPlane* saved_planes;
  int saved_nplanes;
  // umma: every pass on the split-BF16 tensor-core kernel (mixed-precision
  // plans); err: where that kernel records an expired wait (null while only
  // sizing buffers); planes: the plan's matrices with their BF16 pair planes
  // fp32: every pass on the CUDA-core kernel in FP32 arithmetic (FP32 plans)
  explicit AxisPolicy(int min_ctas, int cuda_cores_only = 0, bool umma = false, int* err = nullptr,
                      bool fp32 = false, const UmmaPlane* planes = nullptr, int nplanes = 0)
      : saved(g_axis_min_ctas), saved_mma(g_axis_mma), saved_umma(g_axis_umma), saved_fp32(g_axis_fp32),
        saved_err(g_umma_err), saved_planes(g_umma_planes), saved_nplanes(g_umma_nplanes) {
    g_axis_min_ctas = min_ctas > 0 ? min_ctas : AX_MIN_CTAS;
    g_axis_mma = cuda_cores_only == 0 && !fp32;
    g_axis_umma = umma;
    g_axis_fp32 = fp32;
    g_umma_err = err;
    g_umma_planes = planes;
    g_umma_nplanes = planes ? nplanes : 0;
  }
  ~AxisPolicy() {
    g_axis_min_ctas = saved;
    g_axis_mma = saved_mma;
    g_axis_umma = saved_umma;
    g_axis_fp32 = saved_fp32;
    g_umma_err = saved_err;
    g_umma_planes = saved_planes;
    g_umma_nplanes = saved_nplanes;
  }
};

// The choice depends on (Nout, A, B) only, so axis_blocks() sizes partial
// buffers for exactly the kernel launch_axis() runs.
inline AxisShape axis_shape(int Nout, int A, int B) {
  const int ncol = A * B;
  if (g_axis_umma) {
    const int nc = axu_nc(Nout, ncol);
    return {true, dim3((ncol + nc - 1) / nc, (Nout + AXU_M - 1) / AXU_M), 6};
  }
  if (g_axis_mma && Nout >= 16) {
    // the largest tile that fills one wave (a CTA per SM); else the smallest
    const int tiles[4][2] = {{64, 128}, {64, 64}, {32, 128}, {32, 64}};
    for (int q = 0; q < 4; ++q) {
      const int bm = tiles[q][0], bn = tiles[q][1];
      const dim3 gq((ncol + bn - 1) / bn, (Nout + bm - 1) / bm);
      const long n = (long)gq.x * gq.y;
      if (n >= AXM_SMS || (q == 3 && n >= AXM_MIN_CTAS)) return {true, gq, 2 + q};
    }
  }
  auto grid_of = [&](int ti, int tj) {
    const int tk = (B == 1) ? 16 * tj : 16 * ti;
    const int tc = (B == 1) ? 16 * ti : 16 * tj;
    return dim3((ncol + tc - 1) / tc, (Nout + tk - 1) / tk);
  };
  const dim3 g = grid_of(2, 4);
  if ((long)g.x * g.y >= g_axis_min_ctas) return {true, g, 1};
  return {false, grid_of(1, 1), 0};
}

// Number of CTAs of one pass (the number of partials a reducing epilogue writes).
inline int axis_blocks(int Nout, int A, int B) {
  const AxisShape sh = axis_shape(Nout, A, B);
  return (int)(sh.grid.x * sh.grid.y);
}

// Dynamic shared memory of the tensor-core kernel, raised past the 48 KB
// default once per instantiation.
template <bool CONTIG, int BM, int BN, class Epi>
inline void launch_axis_mma(const double* X, const double* Mat, int Nout, int N, int A, int B, const Epi& epi,
                            dim3 grid, cudaStream_t st) {
  constexpr int bytes = axm_smem_bytes<CONTIG, BM, BN>();
  static const bool attr = [] {
    cudaFuncSetAttribute(k_axis_mma<CONTIG, BM, BN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return true;
  }();
  (void)attr;
  launch_pdl(k_axis_mma<CONTIG, BM, BN, Epi>, grid, AX_THREADS, bytes, st, X, Mat, Nout, N, A, B, epi);
}

template <bool CONTIG, class Epi>
inline void launch_axis_mma_kind(int kind, const double* X, const double* Mat, int Nout, int N, int A, int B,
                                 const Epi& epi, dim3 grid, cudaStream_t st) {
  switch (kind) {
    case 2: launch_axis_mma<CONTIG, 64, 128>(X, Mat, Nout, N, A, B, epi, grid, st); break;
    case 3: launch_axis_mma<CONTIG, 64, 64>(X, Mat, Nout, N, A, B, epi, grid, st); break;
    case 4: launch_axis_mma<CONTIG, 32, 128>(X, Mat, Nout, N, A, B, epi, grid, st); break;
    default: launch_axis_mma<CONTIG, 32, 64>(X, Mat, Nout, N, A, B, epi, grid, st); break;
  }
}

// One pass with Mat of Nout x N (N = contraction length).
template <class Epi>
inline void launch_axis(const double* X, const double* Mat, int Nout, int N, int A, int B,
                        const Epi& epi, cudaStream_t st) {
  const AxisShape sh = axis_shape(Nout, A, B);
  if (sh.kind == 6) {
    if (B == 1) launch_axis_umma<true>(X, Mat, Nout, N, A, B, epi, sh.grid, st);
    else launch_axis_umma<false>(X, Mat, Nout, N, A, B, epi, sh.grid, st);
    return;
  }
  if (sh.kind >= 2) {
    if (B == 1) launch_axis_mma_kind<true>(sh.kind, X, Mat, Nout, N, A, B, epi, sh.grid, st);
    else launch_axis_mma_kind<false>(sh.kind, X, Mat, Nout, N, A, B, epi, sh.grid, st);
    return;
  }
  if (g_axis_fp32) {
    if (B == 1) {
      if (sh.big) launch_pdl(k_axis<true, 2, 4, Epi, float>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
      else launch_pdl(k_axis<true, 1, 1, Epi, float>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
    } else {
      if (sh.big) launch_pdl(k_axis<false, 2, 4, Epi, float>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
      else launch_pdl(k_axis<false, 1, 1, Epi, float>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
    }
    return;
  }
  if (B == 1) {
    if (sh.big) launch_pdl(k_axis<true, 2, 4, Epi>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
    else launch_pdl(k_axis<true, 1, 1, Epi>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
  } else {
    if (sh.big) launch_pdl(k_axis<false, 2, 4, Epi>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
    else launch_pdl(k_axis<false, 1, 1, Epi>, sh.grid, AX_THREADS, 0, st, X, Mat, Nout, N, A, B, epi);
  }
}

// ---------------------------------------------------------------------------
// epilogues
// ---------------------------------------------------------------------------

// out = v * mul (mul = 1 for plain intermediate passes)
struct EpiStore {
  static constexpr int kReduce = 0;
  double* out;
  double mul;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const { out[i] = v * mul; }
};

// out += v * mul (accumulate a face source into a face state)
struct EpiAdd {
  static constexpr int kReduce = 0;
  double* out;
  double mul;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const { out[i] += v * mul; }
};

// out = v / div (reconstruct_volume: IDCT_II(a) / sqrt_dV, spectral_ops.py:83-91)
struct EpiDiv {
  static constexpr int kReduce = 0;
  double* out;
  double div;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const { out[i] = v / div; }
};

// Grid-mode latent source at the reconstructed field:
// T = IDCT(a)/sqrt_dV; Q = latent(T, T_prev) (spectral_ops.py:270-289).
struct EpiLatent {
  static constexpr int kReduce = 0;
  PointPhys P;
  const double* Tprev;
  double* Q;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double T = v / P.sqrt_dV;
    Q[i] = latent_source(P, T, ld_in(Tprev + i));
  }
};

// T = IDCT(a_trial)/sqrt_dV and k'(T) for the correction stencil
// (spectral_ops.py:142-148).
struct EpiTemperatureKp {
  static constexpr int kReduce = 0;
  PointPhys P;
  double* T;
  double* kp;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double t = v / P.sqrt_dV;
    T[i] = t;
    kp[i] = k_prime(P, t);
  }
};

// Trial modes after the top-face and latent forcing (solvers/spectral.py:431-443):
//   Qm = q_scale * v; a = aK + KK*Ct[p]*S_top; a += KK*Qm; a += KK*Cb[p]*S_bot
// where v is the last pass of the latent projection: DCT(Q) in grid mode
// (q_scale = sqrt_dV, project_volume) or the box contraction in box mode
// (q_scale = dV_fine, project_box_to_modes). Qm is stored when non-null.
// With RELAX (no property correction) the relaxation of EpiRelax is applied too.
template <bool RELAX>
struct EpiTrial {
  static constexpr int kReduce = RELAX ? 1 : 0;
  PointPhys P;
  const double* aK;
  const double* KK;
  const double* Ct;
  const double* Cb;
  const double* S_top;   // DCT2 of the net top flux, times s_top_scale
  double s_top_scale;
  double q_scale;
  const double* S_bot;   // null when there is no bottom convection
  double* Qm;
  double* a_trial;       // written when !RELAX
  double* a_it;          // read and updated when RELAX
  double* partials;
  int S;                 // ny nx
  double omega;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red& r) const {
    const int z = i / S, yx = i - z * S;
    const double q = v * q_scale;
    if (Qm) Qm[i] = q;
    const double kk = ld_in(KK + i);
    double t = ld_in(aK + i) + kk * ld_in(Ct + z) * (s_top_scale * ld_in(S_top + yx));
    t += kk * q;
    if (S_bot) t += kk * ld_in(Cb + z) * ld_in(S_bot + yx);
    if (RELAX) {
      const double old = a_it[i];
      const double res = t - old;
      a_it[i] = st_mode(res * omega + old, P.round32);
      r.s0 = fma(res, res, r.s0);
      r.s1 = fma(old, old, r.s1);
    } else {
      a_trial[i] = st_mode(t, P.round32);
    }
  }
};

// Property correction and relaxation (solvers/spectral.py:448-468):
//   C = sqrt_dV * DCT(f); a_raw = a_trial + KK*C; res = a_raw - a_old;
//   a = res*omega + a_old; partial sums of res^2 and a_old^2.
struct EpiRelax {
  static constexpr int kReduce = 1;
  PointPhys P;
  const double* a_trial;
  const double* KK;
  double* a_it;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red& r) const {
    const double c = v * P.sqrt_dV;
    const double raw = ld_in(a_trial + i) + ld_in(KK + i) * c;
    const double old = a_it[i];
    const double res = raw - old;
    a_it[i] = st_mode(res * P.omega + old, P.round32);
    r.s0 = fma(res, res, r.s0);
    r.s1 = fma(old, old, r.s1);
  }
};

// Face: T_s = recon_scale * IDCT2(A) then evaporation, convection and the
// optional k_bar/k(T_s) rescale of the net top flux (solvers/spectral.py:388-407).
struct EpiTopFlux {
  static constexpr int kReduce = 0;
  PointPhys P;
  const double* q_las;
  double* q_evap;
  double* q_net;
  int rescale;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double Ts = P.recon_scale * v;
    const double qe = evaporation(P, Ts);
    q_evap[i] = qe;
    const double qc = P.has_top_conv ? P.h_top * (Ts - P.T0) : 0.0;
    double q = ld_in(q_las + i) - qe - qc;
    if (rescale) q = q * (P.kbar / k_blended(P, Ts));
    q_net[i] = q;
  }
};

// Face: convective flux q = -h (T - T0) from a reconstructed face temperature,
// optionally rescaled by k_bar/k(T) (solvers/spectral.py:335-379).
struct EpiConvFace {
  static constexpr int kReduce = 0;
  PointPhys P;
  double h;
  int rescale;
  double* q;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double T = P.recon_scale * v;
    double qc = -h * (T - P.T0);
    if (rescale) qc = qc * (P.kbar / k_blended(P, T));
    q[i] = qc;
  }
};

// Face: plain reconstruction T = recon_scale * IDCT2(A) into out.
struct EpiFaceTemperature {
  static constexpr int kReduce = 0;
  PointPhys P;
  double* out;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    out[i] = P.recon_scale * v;
  }
};

// Face at commit: T_temp = recon_scale * IDCT2(A) with its max
// (solvers/spectral.py:502, 537) and the q_evap_old <- q_evap copy (:512).
struct EpiCommitSurface {
  static constexpr int kReduce = 2;
  PointPhys P;
  double* T_surf;
  const double* q_evap;
  double* q_evap_old;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red& r) const {
    const double T = P.recon_scale * v;
    T_surf[i] = T;
    q_evap_old[i] = q_evap[i];
    r.mx = fmax(r.mx, T);
  }
};

// z-pass of IDCT3(a_old) with one extra output row (Mat row nz = recon_scale *
// Ct[p]): rows k < nz give the cell-centred field, T = v / sqrt_dV, and the
// latent source Q = latent(T, T_prev) (spectral_ops.py:270-289); row nz gives
// the top-surface temperature T_s of the same modes (the 2-D IDCT commutes
// with the z-weighted sum of reconstruct_surface_temperature,
// spectral_ops.py:210-219) and the evaporation / convection / rescaled net
// top flux (solvers/spectral.py:388-407), stored as slab nz of Q so that the
// following DCT3(Q) x- and y-passes also produce DCT2(q_net).
struct EpiLatentSurface {
  static constexpr int kReduce = 0;
  PointPhys P;
  const double* Tprev;
  double* Q;             // (nz + 1) slabs
  const double* q_las;
  double* q_evap;
  int rescale;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int k, int b, double v, Red&) const {
    if (k < P.nz) {
      Q[i] = latent_source(P, v / P.sqrt_dV, ld_in(Tprev + i));
    } else {
      const double Ts = v;
      const double qe = evaporation(P, Ts);
      q_evap[b] = qe;
      const double qc = P.has_top_conv ? P.h_top * (Ts - P.T0) : 0.0;
      double q = ld_in(q_las + b) - qe - qc;
      if (rescale) q = q * (P.kbar / k_blended(P, Ts));
      Q[i] = q;
    }
  }
};

// Commit: z-pass of IDCT3(a) with the extra surface row. Rows k < nz give
// T_prev = IDCT3(a)/sqrt_dV (solvers/spectral.py:520-521); row nz gives the
// surface temperature of the committed modes with its max (:502, :537) and
// the q_evap_old <- q_evap copy (:512).
struct EpiCommitVolume {
  static constexpr int kReduce = 2;
  PointPhys P;
  double* Tprev;
  double* T_surf;
  const double* q_evap;
  double* q_evap_old;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int k, int b, double v, Red& r) const {
    if (k < P.nz) {
      Tprev[i] = v / P.sqrt_dV;
    } else {
      T_surf[b] = v;
      q_evap_old[b] = q_evap[b];
      r.mx = fmax(r.mx, v);
    }
  }
};

// ---- box mode (latent heat on the laser-following fine box) ----
// The box passes contract the modes against the cosine bases of the fine
// cells: T_box = sum a[p][n][m] Bz[p][l] By[n][k] Bx[m][j] with no further
// scale (reconstruct_temperature_box, physics/spectral_ops.py:173-179).

// First step only (initialize_latent_heat_if_needed,
// physics/spectral_ops.py:182-194): T_prev = T_box(aK), Q_prev = 0.
struct EpiBoxInit {
  static constexpr int kReduce = 0;
  const Ctrl* ctrl;
  double* Tprev;
  double* Qprev;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    if (ctrl->have_tprev) return;
    Tprev[i] = v;
    Qprev[i] = 0.0;
  }
};

// Picard iteration: the latent source on the box from the current iterate and
// the shifted history (compute_latent_heat_source, physics/spectral_ops.py:234-267).
// The constant-property source (spectral_cpu_kernels.py:115-140) uses the
// scalars held by value; the blended-rho form (model != 0) reads P.
struct EpiBoxLatent {
  static constexpr int kReduce = 0;
  PointPhys P;
  const double* Tprev;
  double* Q;
  double* partials;
  int model;             // P.latent_model
  double T_solidus, band_inv, latent_factor;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double tp = ld_in(Tprev + i);
    if (model) {
      Q[i] = latent_source(P, v, tp);
      return;
    }
    double fc = (v - T_solidus) * band_inv;
    fc = fc < 0.0 ? 0.0 : (fc > 1.0 ? 1.0 : fc);
    double fp = (tp - T_solidus) * band_inv;
    fp = fp < 0.0 ? 0.0 : (fp > 1.0 ? 1.0 : fp);
    Q[i] = latent_factor * (fc - fp);
  }
};

// Commit (update_latent_heat_history, physics/spectral_ops.py:197-207, and
// solvers/spectral.py:528-533): T_prev = T_box(a); Q_prev = the source of the
// last Picard iteration, or the shifted history when no iteration ran.
struct EpiBoxCommit {
  static constexpr int kReduce = 0;
  const Ctrl* ctrl;
  double* Tprev;
  double* Qprev;
  const double* Qlast;
  const double* Qshift;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    Tprev[i] = v;
    Qprev[i] = ld_in((ctrl->iter > 0 ? Qlast : Qshift) + i);
  }
};

}  // namespace sgh
