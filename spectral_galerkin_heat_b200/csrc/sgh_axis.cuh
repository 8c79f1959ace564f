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
#include "sgh_device.cuh"

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
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// 16 x 16 threads; each owns a TI (slow) x TJ (fast) register tile. The fast
// thread index runs along the contiguous output dimension: k when B == 1
// (CONTIG), c otherwise. Mat and X panels stream through an AX_STAGES-deep
// cp.async pipeline of AX_BK-slice stages (out-of-range elements zero-filled).
// Computes the output tile at (c0, k0) and hands every element to epi; the
// caller reduces r over the block.
template <bool CONTIG, int TI, int TJ, class Epi>
__device__ __forceinline__ void axis_tile(const double* __restrict__ X, const double* __restrict__ Mat,
                                          int Nout, int N, int A, int B, int c0, int k0, const Epi& epi,
                                          Red& r) {
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

  double acc[TI][TJ];
#pragma unroll
  for (int i = 0; i < TI; ++i)
#pragma unroll
    for (int j = 0; j < TJ; ++j) acc[i][j] = 0.0;

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
      double m[CONTIG ? TJ : TI], x[CONTIG ? TI : TJ];
      if (CONTIG) {
#pragma unroll
        for (int j = 0; j < TJ; ++j) m[j] = Ms[stg][kk][f + 16 * j];
#pragma unroll
        for (int i = 0; i < TI; ++i) x[i] = Xs[stg][kk][TI * s + i];
#pragma unroll
        for (int i = 0; i < TI; ++i)
#pragma unroll
          for (int j = 0; j < TJ; ++j) acc[i][j] = fma(m[j], x[i], acc[i][j]);
      } else {
#pragma unroll
        for (int i = 0; i < TI; ++i) m[i] = Ms[stg][kk][TI * s + i];
#pragma unroll
        for (int j = 0; j < TJ; ++j) x[j] = Xs[stg][kk][f + 16 * j];
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
        epi(idx, k, b, acc[i][j], r);
      }
    }
  }
}

template <bool CONTIG, int TI, int TJ, class Epi>
__global__ void __launch_bounds__(AX_THREADS)
k_axis(const double* __restrict__ X, const double* __restrict__ Mat, int Nout, int N, int A, int B,
       Epi epi) {
  constexpr int TK = CONTIG ? 16 * TJ : 16 * TI;
  constexpr int TC = CONTIG ? 16 * TI : 16 * TJ;
  __shared__ double red_sh[2 * (AX_THREADS / 32)];
  Red r;
  axis_tile<CONTIG, TI, TJ>(X, Mat, Nout, N, A, B, blockIdx.x * TC, blockIdx.y * TK, epi, r);
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

// Launch shape of one pass: the 2 x 4 thread tile when it yields enough CTAs
// to cover the SMs, else the 1 x 1 tile (small faces, short axes).
struct AxisShape {
  bool big;
  dim3 grid;
};
constexpr int AX_MIN_CTAS = 132;
// Tile policy of the calling thread: 2 x 4 tiles when that grid has at least
// this many CTAs. Set for the duration of a plan's call by AxisPolicy, so the
// captured graph, eager launches and the partial-buffer sizing agree.
inline thread_local int g_axis_min_ctas = AX_MIN_CTAS;

struct AxisPolicy {
  int saved;
  explicit AxisPolicy(int min_ctas) : saved(g_axis_min_ctas) {
    g_axis_min_ctas = min_ctas > 0 ? min_ctas : AX_MIN_CTAS;
  }
  ~AxisPolicy() { g_axis_min_ctas = saved; }
};

inline AxisShape axis_shape(int Nout, int A, int B) {
  const int ncol = A * B;
  auto grid_of = [&](int ti, int tj) {
    const int tk = (B == 1) ? 16 * tj : 16 * ti;
    const int tc = (B == 1) ? 16 * ti : 16 * tj;
    return dim3((ncol + tc - 1) / tc, (Nout + tk - 1) / tk);
  };
  const dim3 g = grid_of(2, 4);
  if ((long)g.x * g.y >= g_axis_min_ctas) return {true, g};
  return {false, grid_of(1, 1)};
}

// Number of CTAs of one pass (the number of partials a reducing epilogue writes).
inline int axis_blocks(int Nout, int A, int B) {
  const AxisShape sh = axis_shape(Nout, A, B);
  return (int)(sh.grid.x * sh.grid.y);
}

// One pass with Mat of Nout x N (N = contraction length).
template <class Epi>
inline void launch_axis(const double* X, const double* Mat, int Nout, int N, int A, int B,
                        const Epi& epi, cudaStream_t st) {
  const AxisShape sh = axis_shape(Nout, A, B);
  if (B == 1) {
    if (sh.big) k_axis<true, 2, 4, Epi><<<sh.grid, AX_THREADS, 0, st>>>(X, Mat, Nout, N, A, B, epi);
    else k_axis<true, 1, 1, Epi><<<sh.grid, AX_THREADS, 0, st>>>(X, Mat, Nout, N, A, B, epi);
  } else {
    if (sh.big) k_axis<false, 2, 4, Epi><<<sh.grid, AX_THREADS, 0, st>>>(X, Mat, Nout, N, A, B, epi);
    else k_axis<false, 1, 1, Epi><<<sh.grid, AX_THREADS, 0, st>>>(X, Mat, Nout, N, A, B, epi);
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
  const DevParams* P;
  const double* Tprev;
  double* Q;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double T = v / P->sqrt_dV;
    Q[i] = latent_source(*P, T, Tprev[i]);
  }
};

// T = IDCT(a_trial)/sqrt_dV and k'(T) for the correction stencil
// (spectral_ops.py:142-148).
struct EpiTemperatureKp {
  static constexpr int kReduce = 0;
  const DevParams* P;
  double* T;
  double* kp;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double t = v / P->sqrt_dV;
    T[i] = t;
    kp[i] = k_prime(*P, t);
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
  const DevParams* P;
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
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red& r) const {
    const int S = P->S;
    const int z = i / S, yx = i - z * S;
    const double q = v * q_scale;
    if (Qm) Qm[i] = q;
    const double kk = KK[i];
    double t = aK[i] + kk * Ct[z] * (s_top_scale * S_top[yx]);
    t += kk * q;
    if (S_bot) t += kk * Cb[z] * S_bot[yx];
    if (RELAX) {
      const double old = a_it[i];
      const double res = t - old;
      a_it[i] = res * P->omega + old;
      r.s0 = fma(res, res, r.s0);
      r.s1 = fma(old, old, r.s1);
    } else {
      a_trial[i] = t;
    }
  }
};

// Property correction and relaxation (solvers/spectral.py:448-468):
//   C = sqrt_dV * DCT(f); a_raw = a_trial + KK*C; res = a_raw - a_old;
//   a = res*omega + a_old; partial sums of res^2 and a_old^2.
struct EpiRelax {
  static constexpr int kReduce = 1;
  const DevParams* P;
  const double* a_trial;
  const double* KK;
  double* a_it;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red& r) const {
    const double c = v * P->sqrt_dV;
    const double raw = a_trial[i] + KK[i] * c;
    const double old = a_it[i];
    const double res = raw - old;
    a_it[i] = res * P->omega + old;
    r.s0 = fma(res, res, r.s0);
    r.s1 = fma(old, old, r.s1);
  }
};

// Face: T_s = recon_scale * IDCT2(A) then evaporation, convection and the
// optional k_bar/k(T_s) rescale of the net top flux (solvers/spectral.py:388-407).
struct EpiTopFlux {
  static constexpr int kReduce = 0;
  const DevParams* P;
  const double* q_las;
  double* q_evap;
  double* q_net;
  int rescale;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double Ts = P->recon_scale * v;
    const double qe = evaporation(*P, Ts);
    q_evap[i] = qe;
    const double qc = P->has_top_conv ? P->h_top * (Ts - P->T0) : 0.0;
    double q = q_las[i] - qe - qc;
    if (rescale) q = q * (P->kbar / k_blended(*P, Ts));
    q_net[i] = q;
  }
};

// Face: convective flux q = -h (T - T0) from a reconstructed face temperature,
// optionally rescaled by k_bar/k(T) (solvers/spectral.py:335-379).
struct EpiConvFace {
  static constexpr int kReduce = 0;
  const DevParams* P;
  double h;
  int rescale;
  double* q;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    const double T = P->recon_scale * v;
    double qc = -h * (T - P->T0);
    if (rescale) qc = qc * (P->kbar / k_blended(*P, T));
    q[i] = qc;
  }
};

// Face: plain reconstruction T = recon_scale * IDCT2(A) into out.
struct EpiFaceTemperature {
  static constexpr int kReduce = 0;
  const DevParams* P;
  double* out;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    out[i] = P->recon_scale * v;
  }
};

// Face at commit: T_temp = recon_scale * IDCT2(A) with its max
// (solvers/spectral.py:502, 537) and the q_evap_old <- q_evap copy (:512).
struct EpiCommitSurface {
  static constexpr int kReduce = 2;
  const DevParams* P;
  double* T_surf;
  const double* q_evap;
  double* q_evap_old;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red& r) const {
    const double T = P->recon_scale * v;
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
  const DevParams* P;
  const double* Tprev;
  double* Q;             // (nz + 1) slabs
  const double* q_las;
  double* q_evap;
  int rescale;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int k, int b, double v, Red&) const {
    if (k < P->nz) {
      Q[i] = latent_source(*P, v / P->sqrt_dV, Tprev[i]);
    } else {
      const double Ts = v;
      const double qe = evaporation(*P, Ts);
      q_evap[b] = qe;
      const double qc = P->has_top_conv ? P->h_top * (Ts - P->T0) : 0.0;
      double q = q_las[b] - qe - qc;
      if (rescale) q = q * (P->kbar / k_blended(*P, Ts));
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
  const DevParams* P;
  double* Tprev;
  double* T_surf;
  const double* q_evap;
  double* q_evap_old;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int k, int b, double v, Red& r) const {
    if (k < P->nz) {
      Tprev[i] = v / P->sqrt_dV;
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
struct EpiBoxLatent {
  static constexpr int kReduce = 0;
  const DevParams* P;
  const double* Tprev;
  double* Q;
  double* partials;
  __device__ __forceinline__ void operator()(int i, int, int, double v, Red&) const {
    Q[i] = latent_source(*P, v, Tprev[i]);
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
    Qprev[i] = ctrl->iter > 0 ? Qlast[i] : Qshift[i];
  }
};

}  // namespace sgh
