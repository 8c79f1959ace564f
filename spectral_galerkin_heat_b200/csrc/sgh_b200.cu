// sgh_b200.cu -- libsgh_b200.so: the spectral-Galerkin heat time step on B200.
//
// One plan = one cuboid instance. sgh_plan_bind() builds every table on the
// device and captures the whole time step -- laser/face forcing, ETD1 update,
// the Picard fixed-point loop and the commit -- into ONE CUDA graph:
//
//   G:  while (step < n_target) {                      <- conditional node
//         step_begin, face forcing, initial guess, convection guesses
//         while (Picard not converged and iter < cap) { <- conditional node
//           surface reconstruction + evaporation / convection face flux
//           [latent: IDCT3 -> latent source -> DCT3]  (fused epilogues)
//           [property correction: IDCT3 -> k' -> stencil -> DCT3]
//           relaxation + residual norms, convergence test on the device
//         }
//         commit: surface max, history buffers, metrics
//       }
//
// so a step (or a batch of steps) costs one graph launch and no host
// synchronisation per Picard iteration, where the reference issues ~20 array
// operations and one device->host float() per iteration
// (solvers/spectral.py:386-499).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sgh_axis.cuh"
#include "sgh_b200.h"
#include "sgh_device.cuh"

namespace {
thread_local std::string g_last_error;
}  // namespace

int sgh::set_error(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

using namespace sgh;

namespace {

thread_local int g_launches = 0;  // kernels enqueued by the enqueue_* helpers

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define SGH_CK(call)                                                                      \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(SGH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// In the void enqueue helpers a failed async call is reported by the
// cudaGetLastError / capture-end checks of the caller.
#define SGH_CK_VOID(call) (void)(call)

constexpr int EW_THREADS = 256;

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------

// Orthonormal DCT-II matrix C[k][n] = w_k cos(pi k (2n+1) / (2N)) and its
// transpose. The angle is reduced exactly in integers (period 4N) before cospi.
__global__ void k_dct_matrix(int N, double* M, double* MT) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * N) return;
  const int k = e / N, n = e - k * N;
  const long long m = ((long long)k * (2 * n + 1)) % (4LL * N);
  const double w = (k == 0) ? sqrt(1.0 / N) : sqrt(2.0 / N);
  const double v = w * cospi((double)m / (double)(2 * N));
  M[k * N + n] = v;
  MT[n * N + k] = v;
}

// Propagators exactly as precompute_K_KK (physics/spectral_state.py:374-421):
// lam = alpha ((kz^2 + ky^2) + kx^2), K = exp(-lam dt), KK = (K - 1)/(-lam)/(rho c),
// KK[0,0,0] = dt/(rho c).
__global__ void k_propagators(const DevParams* __restrict__ P, double alpha, double rho_cp,
                              double* K, double* KK) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P->V) return;
  const int S = P->S, nx = P->nx;
  const int z = i / S, r = i - z * S, y = r / nx, x = r - y * nx;
  const double kz = M_PI * (double)z / P->Lz;
  const double ky = M_PI * (double)y / P->Ly;
  const double kx = M_PI * (double)x / P->Lx;
  const double lam = alpha * (kz * kz + ky * ky + kx * kx);
  const double k = exp(-lam * P->dt);
  K[i] = k;
  KK[i] = (i == 0) ? P->dt / rho_cp : ((k - 1.0) / (-lam)) / rho_cp;
}

// Cell-centred coordinates and the top / bottom z-weights
// (SpectralGrid, physics/spectral_state.py:98-122; _C_coef spectral_helpers.py:26-46).
// Also appends to the inverse z-matrix MzT (nz x nz) the rows recon_scale *
// Ct[p] (top) and recon_scale * Cb[p] (bottom), so that an inverse z-pass
// yields the surface temperatures beside the cell-centred field.
__global__ void k_grid_tables(const DevParams* __restrict__ P, double* xc, double* yc, double* Ct,
                              double* Cb, double* MzT_aug) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P->nx) xc[i] = ((double)i + 0.5) * P->dx;
  if (i < P->ny) yc[i] = ((double)i + 0.5) * P->dy;
  if (i < P->nz) {
    const int nz = P->nz;
    const double c = (i == 0) ? sqrt(1.0 / P->Lz) : sqrt(2.0 / P->Lz);
    const double ct = (i & 1) ? -c : c;
    Cb[i] = c;
    Ct[i] = ct;
    MzT_aug[(size_t)nz * nz + i] = P->recon_scale * ct;
    MzT_aug[(size_t)(nz + 1) * nz + i] = P->recon_scale * c;
  }
}

// Initial condition (solvers/spectral.py:176-202).
__global__ void k_reset(const DevParams* __restrict__ P, Ctrl* ctrl, double* a, double* Tprev,
                        double* q_evap_old, double* q_evap, double* Qm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P->V) {
    a[i] = (i == 0) ? P->T0 * sqrt(P->Lx * P->Ly * P->Lz) : 0.0;
    Tprev[i] = P->T0;
    Qm[i] = 0.0;
  }
  if (i < P->S) {
    q_evap_old[i] = 0.0;
    q_evap[i] = 0.0;
  }
  if (i == 0) {
    ctrl->have_qprev = 0;
    ctrl->step = 0;
    ctrl->n_target = 0;
    ctrl->have_tprev = 0;
    ctrl->box_i0x = -1;
    ctrl->box_i0y = -1;
  }
}

// Warm-start flags of a restored state (sgh_state_set_flags).
__global__ void k_set_flags(Ctrl* ctrl, int flags) {
  ctrl->have_qprev = (flags & SGH_STATE_HAVE_Q_MODES) ? 1 : 0;
  ctrl->have_tprev = (flags & SGH_STATE_HAVE_BOX) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// box mode: tables, window, history
// ---------------------------------------------------------------------------

// Fine-cell cosine bases (FineMeshState.__init__, physics/spectral_state.py:194-219):
// B[m][i] = C_m cos(pi m c_i / L) at the fine cell centres c_i = z0 + (i + 0.5) d
// (z0 = 0 for x and y, Lz - Lz_box for z), C_m = sqrt(1/L), sqrt(2/L)
// (physics/spectral_helpers.py:26-46). Written point-major, T[i][m] (the
// matrix of a reconstruction pass), and, when F is non-null, mode-major
// F[m][i] (the matrix of a projection pass).
__global__ void k_fine_basis(int n_modes, int n_pts, double L, double d, double z0, double* T, double* F) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n_modes * n_pts) return;
  const int i = (int)(e / n_modes), m = (int)(e - (long long)i * n_modes);
  const double c = (m == 0) ? sqrt(1.0 / L) : sqrt(2.0 / L);
  const double coord = z0 + ((double)i + 0.5) * d;
  const double v = c * cos(((M_PI * (double)m) * coord) / L);
  T[e] = v;
  if (F) F[(size_t)m * n_pts + i] = v;
}

// Start of the window of n_box fine cells centred on pos, clamped to the fine
// grid (_calculate_subgrid_indices, physics/spectral_helpers.py:49-85).
// Python's round() rounds half to even, as rint() does.
__device__ int box_start(double q, int n_total, int n_box) {
  const double g = rint(fmax(0.0, fmin(q, (double)(n_total - 1))));
  long long st = (long long)g - n_box / 2;
  const long long max_start = n_total > n_box ? n_total - n_box : 0;
  if (st > max_start) st = max_start;
  if (st < 0) st = 0;
  return (int)st;
}

// Window bases of this step (FineMeshState.update, physics/spectral_state.py:229-237):
// rows i0 .. i0 + n_box - 1 of the point-major x and y tables, stored for the
// reconstruction passes (Wi, n_box x n) and the projection passes (Wf, n x n_box).
__global__ void __launch_bounds__(EW_THREADS)
k_box_window(const DevParams* __restrict__ P, const Ctrl* __restrict__ ctrl, const double* __restrict__ BxT,
             const double* __restrict__ ByT, double* Wxi, double* Wxf, double* Wyi, double* Wyf) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nX = (long long)P->xb * P->nx;
  if (e < nX) {
    const int j = (int)(e / P->nx), m = (int)(e - (long long)j * P->nx);
    const double v = BxT[(size_t)(ctrl->box_i0x + j) * P->nx + m];
    Wxi[e] = v;
    Wxf[(size_t)m * P->xb + j] = v;
    return;
  }
  const long long f = e - nX;
  if (f < (long long)P->yb * P->ny) {
    const int j = (int)(f / P->ny), n = (int)(f - (long long)j * P->ny);
    const double v = ByT[(size_t)(ctrl->box_i0y + j) * P->ny + n];
    Wyi[f] = v;
    Wyf[(size_t)n * P->yb + j] = v;
  }
}

// First step only: aK = a K, the modes the history is seeded from
// (solvers/spectral.py:283, 292-293).
__global__ void __launch_bounds__(EW_THREADS)
k_box_seed(const DevParams* __restrict__ P, const Ctrl* __restrict__ ctrl, const double* __restrict__ a,
           const double* __restrict__ K, double* aK) {
  if (ctrl->have_tprev) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P->V) aK[i] = a[i] * K[i];
}

// History shift (shift_latent_heat_history, physics/spectral_ops.py:292-306):
// order-1 translation of every z-layer of T_prev ('nearest') and Q_prev
// ('constant', 0 outside) by -v dt / d_fine pixels (the tables of _ndshift,
// physics/spectral_cpu_kernels.py:302-371). Marks the history present.
__global__ void __launch_bounds__(EW_THREADS)
k_box_shift(const DevParams* __restrict__ P, Ctrl* ctrl, const double* __restrict__ Tp,
            const double* __restrict__ Qp, double* Ts, double* Qs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P->Nb) {
    const int xb = P->xb, yb = P->yb, L = xb * yb;
    const int z = i / L, r = i - z * L, y = r / xb, x = r - y * xb;
    const ShiftTap ty = shift_tap(y, yb, ctrl->box_sy);
    const ShiftTap tx = shift_tap(x, xb, ctrl->box_sx);
    const size_t r0 = (size_t)z * L + (size_t)ty.i0 * xb, r1 = (size_t)z * L + (size_t)ty.i1 * xb;
    Ts[i] = ty.w0 * (tx.w0 * Tp[r0 + tx.i0] + tx.w1 * Tp[r0 + tx.i1]) +
            ty.w1 * (tx.w0 * Tp[r1 + tx.i0] + tx.w1 * Tp[r1 + tx.i1]);
    double q = ty.w0 * (tx.w0 * Qp[r0 + tx.i0] + tx.w1 * Qp[r0 + tx.i1]) +
               ty.w1 * (tx.w0 * Qp[r1 + tx.i0] + tx.w1 * Qp[r1 + tx.i1]);
    if (!(ty.in && tx.in)) q = 0.0;
    Qs[i] = q;
  }
  if (i == 0) ctrl->have_tprev = 1;
}

// Magnitude maxima of the committed latent source over the box, its floor
// (z = 0) and its x and y edge columns, for the truncation check
// (SpectralSolver._check_latent_box_truncation, solvers/spectral.py:545-586).
// Skipped when no Picard iteration ran (no source of this step). fmax drops
// NaN sources, where the reference's max would return NaN and flag nothing;
// such a step already reports SGH_STEP_NONFINITE.
__global__ void __launch_bounds__(EW_THREADS)
k_box_check(const DevParams* __restrict__ P, Ctrl* ctrl, const double* __restrict__ Q) {
  if (ctrl->iter <= 0) return;
  const int xb = P->xb, yb = P->yb, L = xb * yb;
  double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P->Nb; i += gridDim.x * blockDim.x) {
    const int z = i / L, r = i - z * L, y = r / xb, x = r - y * xb;
    const double q = fabs(Q[i]);
    m0 = fmax(m0, q);
    if (z == 0) m1 = fmax(m1, q);
    if (x == 0 || x == xb - 1) m2 = fmax(m2, q);
    if (y == 0 || y == yb - 1) m3 = fmax(m3, q);
  }
  for (int o = 16; o > 0; o >>= 1) {
    m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    m3 = fmax(m3, __shfl_xor_sync(0xffffffffu, m3, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&ctrl->box_max[0], (unsigned long long)__double_as_longlong(m0));
    atomicMax(&ctrl->box_max[1], (unsigned long long)__double_as_longlong(m1));
    atomicMax(&ctrl->box_max[2], (unsigned long long)__double_as_longlong(m2));
    atomicMax(&ctrl->box_max[3], (unsigned long long)__double_as_longlong(m3));
  }
}

// ---------------------------------------------------------------------------
// step kernels
// ---------------------------------------------------------------------------

__global__ void k_run_setup(Ctrl* ctrl, sgh_laser laser, const sgh_laser* table, sgh_step_out* outs,
                            int n) {
  ctrl->laser = laser;
  ctrl->table = table;
  ctrl->out_table = outs;
  ctrl->n_target = n;
  ctrl->step = 0;
}

// Laser state of this step, I0 = A P / (f r_x r_y) (core/laser.py:110-112,
// solvers/spectral.py:258-268) and the warm-start shift in pixels
// (spectral_cpu_kernels.py:392-396); opens the Picard loop.
__global__ void k_step_begin(const DevParams* __restrict__ P, Ctrl* ctrl,
                             cudaGraphConditionalHandle h_picard, cudaGraphConditionalHandle h_seed,
                             int in_graph) {
  if (ctrl->table) ctrl->laser = ctrl->table[ctrl->step];
  const sgh_laser L = ctrl->laser;
  ctrl->I0 = L.is_on ? P->absorptivity * L.power / (P->area_factor * (P->r_x * P->r_y)) : 0.0;
  const bool f32 = (L.flags & SGH_LASER_F32) != 0;
  ctrl->shift_x = laser_shift(L.vx, P->dt, P->dx, f32);
  ctrl->shift_y = laser_shift(L.vy, P->dt, P->dy, f32);
  ctrl->iter = 0;
  ctrl->stop = 0;
  ctrl->status = SGH_STEP_CAPPED;
  ctrl->rel_err = nan("");
  if (in_graph) cudaGraphSetConditional(h_picard, P->max_iter > 0 ? 1u : 0u);
  if (P->box) {
    // window of this step and the history shift in fine pixels
    // (physics/spectral_state.py:229-237, physics/spectral_ops.py:300-302)
    ctrl->box_i0x = box_start(laser_cells(L.x, P->dxf, f32), P->fx, P->xb);
    ctrl->box_i0y = box_start(laser_cells(L.y, P->dyf, f32), P->fy, P->yb);
    ctrl->box_sx = -laser_shift(L.vx, P->dt, P->dxf, f32);
    ctrl->box_sy = -laser_shift(L.vy, P->dt, P->dyf, f32);
    for (int j = 0; j < 4; ++j) ctrl->box_max[j] = 0ull;
    if (in_graph) cudaGraphSetConditional(h_seed, ctrl->have_tprev ? 0u : 1u);
  }
}

// Face forcing of the initial guess: q_las, P_laser partials, and
// q_net = q_las - shift(q_evap_old) (solvers/spectral.py:273-306).
__global__ void __launch_bounds__(EW_THREADS)
k_face_begin(const DevParams* __restrict__ P, const Ctrl* __restrict__ ctrl, const double* xc,
             const double* yc, const double* q_evap_old, double* q_las, double* q_net,
             double* partials) {
  __shared__ double sh[2 * (EW_THREADS / 32)];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = P->nx, ny = P->ny;
  double sum = 0.0, dummy = 0.0;
  if (i < P->S) {
    const int y = i / nx, x = i - y * nx;
    const double q = laser_flux(*P, ctrl->I0, ctrl->laser.x, ctrl->laser.y, xc[x], yc[y]);
    q_las[i] = q;
    sum = q;
    const ShiftTap ty = shift_tap(y, ny, ctrl->shift_y);
    const ShiftTap tx = shift_tap(x, nx, ctrl->shift_x);
    double v = ty.w0 * (tx.w0 * q_evap_old[ty.i0 * nx + tx.i0] + tx.w1 * q_evap_old[ty.i0 * nx + tx.i1]) +
               ty.w1 * (tx.w0 * q_evap_old[ty.i1 * nx + tx.i0] + tx.w1 * q_evap_old[ty.i1 * nx + tx.i1]);
    if (!(ty.in && tx.in)) v = 0.0;
    q_net[i] = q - v;
  }
  block_sum2<EW_THREADS>(sum, dummy, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = sum;
}

// A[y,x] = sum_p w[p] a[p,y,x]  (einsum 'p,pij->ij', spectral_ops.py:210-231)
__global__ void __launch_bounds__(EW_THREADS)
k_zsum(const double* __restrict__ a, const double* __restrict__ w, int nz, int S, double* A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  double s = 0.0;
  for (int p = 0; p < nz; ++p) s = fma(w[p], a[(size_t)p * S + i], s);
  A[i] = s;
}

// a <- K a; a_temp = aK + KK Ct[p] S_top [+ KK Q_prev]  (solvers/spectral.py:283, 320-334);
// in box mode Q_prev is the projection of the shifted box history (:323-327).
__global__ void __launch_bounds__(EW_THREADS)
k_init_modes(const DevParams* __restrict__ P, const Ctrl* __restrict__ ctrl, double* a_it,
             const double* __restrict__ K, const double* __restrict__ KK, const double* __restrict__ Ct,
             const double* __restrict__ S_top, const double* __restrict__ Qm, double* aK) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P->V) return;
  const int S = P->S;
  const int z = i / S, yx = i - z * S;
  const double ak = st_mode(a_it[i] * K[i], P->round32);
  aK[i] = ak;
  const double kk = KK[i];
  double t = ak + kk * Ct[z] * S_top[yx];
  if (ctrl->have_qprev || P->box) t += kk * Qm[i];
  a_it[i] = st_mode(t, P->round32);
}

// a += KK w[p] S[y,x]  (add_bottom_surface_source, spectral_cpu_kernels.py:105-113)
__global__ void __launch_bounds__(EW_THREADS)
k_add_face(const DevParams* __restrict__ P, double* a, const double* __restrict__ KK,
           const double* __restrict__ w, const double* __restrict__ Sf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P->V) return;
  const int S = P->S;
  const int z = i / S, yx = i - z * S;
  a[i] = st_mode(a[i] + KK[i] * w[z] * Sf[yx], P->round32);
}

// Trial modes without latent heat (property correction follows).
__global__ void __launch_bounds__(EW_THREADS)
k_trial(const DevParams* __restrict__ P, const double* __restrict__ aK, const double* __restrict__ KK,
        const double* __restrict__ Ct, const double* __restrict__ Cb, const double* __restrict__ S_top,
        const double* __restrict__ S_bot, double* a_trial) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P->V) return;
  const int S = P->S;
  const int z = i / S, yx = i - z * S;
  const double kk = KK[i];
  double t = aK[i] + kk * Ct[z] * S_top[yx];
  if (S_bot) t += kk * Cb[z] * S_bot[yx];
  a_trial[i] = st_mode(t, P->round32);
}

// Trial modes and relaxation in one pass when there is neither latent heat nor
// property correction (solvers/spectral.py:431-468).
constexpr int RELAX_BLOCKS_MAX = 1184;  // 8 x 148 SMs
__global__ void __launch_bounds__(EW_THREADS)
k_trial_relax(const DevParams* __restrict__ P, const double* __restrict__ aK,
              const double* __restrict__ KK, const double* __restrict__ Ct,
              const double* __restrict__ Cb, const double* __restrict__ S_top,
              const double* __restrict__ S_bot, double* a_it, double* partials) {
  __shared__ double sh[2 * (EW_THREADS / 32)];
  const int S = P->S, V = P->V;
  const double om = P->omega;
  double s0 = 0.0, s1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    const int z = i / S, yx = i - z * S;
    const double kk = KK[i];
    double t = aK[i] + kk * Ct[z] * S_top[yx];
    if (S_bot) t += kk * Cb[z] * S_bot[yx];
    const double old = a_it[i];
    const double res = t - old;
    a_it[i] = st_mode(res * om + old, P->round32);
    s0 = fma(res, res, s0);
    s1 = fma(old, old, s1);
  }
  block_sum2<EW_THREADS>(s0, s1, sh);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = s0;
    partials[2 * blockIdx.x + 1] = s1;
  }
}

// f = div(k' grad T) - a'(T) (T - T_prev)/dt with the numpy.gradient
// (edge_order=1) stencil applied twice (spectral_cpu_kernels.py:165-252).
__global__ void __launch_bounds__(EW_THREADS)
k_stencil(const DevParams* __restrict__ P, const double* __restrict__ T, const double* __restrict__ kp,
          const double* __restrict__ Tprev, double* f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P->V) return;
  const int nx = P->nx, ny = P->ny, nz = P->nz, S = P->S;
  const int z = i / S, r = i - z * S, y = r / nx, x = r - y * nx;
  const double idx = P->inv_dx, idy = P->inv_dy, idz = P->inv_dz;

  // g along one axis at position q (stride st, extent n, base offset b0 of the line)
  auto g_at = [&](int q, int n, int st, int b0, double inv) -> double {
    double d;
    if (q == 0) d = (T[b0 + st] - T[b0]) * inv;
    else if (q == n - 1) d = (T[b0 + (n - 1) * st] - T[b0 + (n - 2) * st]) * inv;
    else d = (T[b0 + (q + 1) * st] - T[b0 + (q - 1) * st]) * (0.5 * inv);
    return kp[b0 + q * st] * d;
  };
  auto div_axis = [&](int q, int n, int st, int b0, double inv) -> double {
    if (q == 0) return (g_at(1, n, st, b0, inv) - g_at(0, n, st, b0, inv)) * inv;
    if (q == n - 1) return (g_at(n - 1, n, st, b0, inv) - g_at(n - 2, n, st, b0, inv)) * inv;
    return (g_at(q + 1, n, st, b0, inv) - g_at(q - 1, n, st, b0, inv)) * (0.5 * inv);
  };
  const double dgx = div_axis(x, nx, 1, z * S + y * nx, idx);
  const double dgy = div_axis(y, ny, nx, z * S + x, idy);
  const double dgz = div_axis(z, nz, S, r, idz);
  const double t = T[i];
  const double dTdt = (t - Tprev[i]) * P->inv_dt;
  f[i] = dgx + dgy + dgz - a_prime(*P, t) * dTdt;
}

// Convergence test of one Picard iteration (solvers/spectral.py:464-499):
// err = sqrt(sum res^2 / n) / max(sqrt(sum a_old^2 / n), 1e-9).
__global__ void __launch_bounds__(EW_THREADS)
k_converge(const DevParams* __restrict__ P, Ctrl* ctrl, const double* __restrict__ partials,
           int nparts, const double* __restrict__ extra_old, int n_extra,
           cudaGraphConditionalHandle h_picard, int in_graph) {
  __shared__ double sh[2 * (EW_THREADS / 32)];
  double s0 = 0.0, s1 = 0.0;
  for (int b = threadIdx.x; b < nparts; b += EW_THREADS) {
    s0 += partials[2 * b];
    s1 += partials[2 * b + 1];
  }
  for (int b = threadIdx.x; b < n_extra; b += EW_THREADS) s1 += extra_old[b];
  block_sum2<EW_THREADS>(s0, s1, sh);
  if (threadIdx.x == 0) {
    const double n = P->n_elements;
    const double rms_d = sqrt(s0 / n);
    const double rms_o = sqrt(s1 / n);
    const double rel = rms_d / fmax(rms_o, 1e-9);
    const int it = ctrl->iter + 1;
    ctrl->iter = it;
    ctrl->rel_err = rel;
    if (ctrl->hist && it <= ctrl->hist_cap) {
      ctrl->hist[2 * (it - 1)] = rms_d;
      ctrl->hist[2 * (it - 1) + 1] = rel;
    }
    int stop = 0;
    if (rel < P->tol) {
      ctrl->status = SGH_STEP_CONVERGED;
      stop = 1;
    } else if (!isfinite(rel)) {
      ctrl->status = SGH_STEP_NONFINITE;
      stop = 1;
    } else if (it >= P->max_iter) {
      ctrl->status = SGH_STEP_CAPPED;
      stop = 1;
    }
    ctrl->stop = stop;
    if (in_graph) cudaGraphSetConditional(h_picard, stop ? 0u : 1u);
  }
}

// Where k_converge records the Picard history of a step.
__global__ void k_ctrl_history(Ctrl* ctrl, double* hist, int cap) {
  ctrl->hist = hist;
  ctrl->hist_cap = cap;
}

// Metrics and history of the committed step (solvers/spectral.py:502-542);
// advances the step counter and decides whether the step loop continues.
__global__ void __launch_bounds__(EW_THREADS)
k_commit(const DevParams* __restrict__ P, Ctrl* ctrl, const double* __restrict__ las_parts,
         int n_las, const double* __restrict__ surf_parts, int n_surf,
         cudaGraphConditionalHandle h_steps, int in_graph) {
  __shared__ double sh[2 * (EW_THREADS / 32)];
  double s = 0.0, d = 0.0;
  for (int b = threadIdx.x; b < n_las; b += EW_THREADS) s += las_parts[b];
  block_sum2<EW_THREADS>(s, d, sh);
  double m = -INFINITY, d2 = 0.0;
  for (int b = threadIdx.x; b < n_surf; b += EW_THREADS) m = fmax(m, surf_parts[2 * b]);
  block_max_sum<EW_THREADS>(m, d2, sh);
  if (threadIdx.x == 0) {
    sgh_step_out o;
    o.T_surface_max = m;
    o.P_laser = s * P->dx * P->dy;
    o.picard_rel_err = ctrl->rel_err;
    o.n_iter = ctrl->iter;
    o.converged = ctrl->status == SGH_STEP_CONVERGED ? 1 : 0;
    o.status = ctrl->umma_err ? SGH_STEP_TC_TIMEOUT : ctrl->status;
    int flags = 0;
    if (P->box && ctrl->iter > 0) {
      // truncation check (solvers/spectral.py:545-586): a face of the box whose
      // source exceeds 1% of the peak; x and y only where the box is a window
      const double peak = __longlong_as_double((long long)ctrl->box_max[0]);
      if (peak > 0.0) {
        const double thr = 1e-2 * peak;
        if (__longlong_as_double((long long)ctrl->box_max[1]) > thr) flags |= SGH_STEP_FLAG_BOX_FLOOR;
        if (P->xb < P->fx && __longlong_as_double((long long)ctrl->box_max[2]) > thr) flags |= SGH_STEP_FLAG_BOX_X;
        if (P->yb < P->fy && __longlong_as_double((long long)ctrl->box_max[3]) > thr) flags |= SGH_STEP_FLAG_BOX_Y;
      }
    }
    o.flags = flags;
    ctrl->out = o;
    if (ctrl->out_table) ctrl->out_table[ctrl->step] = o;
    if (P->grid_latent && P->max_iter > 0) ctrl->have_qprev = 1;
    const int next = ctrl->step + 1;
    ctrl->step = next;
    if (in_graph) cudaGraphSetConditional(h_steps, next < ctrl->n_target ? 1u : 0u);
  }
}

// ---------------------------------------------------------------------------
// face-space Picard (no latent heat, no property correction)
// ---------------------------------------------------------------------------
// Without the volume forcing terms every iterate of the step is
//   a_it = aK + KK (Ct[p] sigma[y,x] + Cb[p] beta[y,x])
// with face fields sigma (top) and beta (bottom): the initial guess
// (solvers/spectral.py:320-351), each trial (:431-443) and each relaxation
// (:459-462) keep that form. The surface temperatures, the residual and the
// norm of the iterate then reduce to face fields built once per step from the
// modes, and the Picard loop runs on faces only. Per step the volume is read
// twice and written once, whatever the iteration count.

// Constant face weights of KK (bind time):
// W_tt = sum Ct^2 KK, W_tb = sum Ct Cb KK, W_bb = sum Cb^2 KK,
// Q_tt = sum (KK Ct)^2, Q_tb = sum KK^2 Ct Cb, Q_bb = sum (KK Cb)^2.
__global__ void __launch_bounds__(EW_THREADS)
k_fs_weights(const DevParams* __restrict__ P, const double* __restrict__ KK, const double* __restrict__ Ct,
             const double* __restrict__ Cb, double* W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int S = P->S;
  if (i >= S) return;
  double wtt = 0, wtb = 0, wbb = 0, qtt = 0, qtb = 0, qbb = 0;
  for (int p = 0; p < P->nz; ++p) {
    const double kk = KK[(size_t)p * S + i], ct = Ct[p], cb = Cb[p];
    wtt += ct * ct * kk;
    wtb += ct * cb * kk;
    wbb += cb * cb * kk;
    qtt += (kk * ct) * (kk * ct);
    qtb += kk * kk * ct * cb;
    qbb += (kk * cb) * (kk * cb);
  }
  W[0 * S + i] = wtt; W[1 * S + i] = wtb; W[2 * S + i] = wbb;
  W[3 * S + i] = qtt; W[4 * S + i] = qtb; W[5 * S + i] = qbb;
}

// Per step: with aK = K a (not stored), the face fields
// Zt = sum Ct aK, Zb = sum Cb aK, Yt = sum aK KK Ct, Yb = sum aK KK Cb, and
// per-CTA partial sums of aK^2. Also opens the face state: sigma = beta = 0.
__global__ void __launch_bounds__(EW_THREADS)
k_fs_pass1(const DevParams* __restrict__ P, const double* __restrict__ a, const double* __restrict__ K,
           const double* __restrict__ KK, const double* __restrict__ Ct, const double* __restrict__ Cb,
           double* F, double* n1_parts) {
  __shared__ double sh[2 * (EW_THREADS / 32)];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int S = P->S;
  double n1 = 0.0, dummy = 0.0;
  if (i < S) {
    double zt = 0, zb = 0, yt = 0, yb = 0;
    for (int p = 0; p < P->nz; ++p) {
      const size_t j = (size_t)p * S + i;
      const double ak = a[j] * K[j];
      const double kk = KK[j];
      zt = fma(Ct[p], ak, zt);
      zb = fma(Cb[p], ak, zb);
      yt = fma(ak * kk, Ct[p], yt);
      yb = fma(ak * kk, Cb[p], yb);
      n1 = fma(ak, ak, n1);
    }
    F[0 * S + i] = zt; F[1 * S + i] = zb; F[2 * S + i] = yt; F[3 * S + i] = yb;
  }
  block_sum2<EW_THREADS>(n1, dummy, sh);
  if (threadIdx.x == 0) n1_parts[blockIdx.x] = n1;
}

// Face inputs of the two surface reconstructions of the current iterate:
// At = Zt + W_tt sigma + W_tb beta (top), Ab = Zb + W_tb sigma + W_bb beta (bottom).
__global__ void __launch_bounds__(EW_THREADS)
k_fs_assemble(const DevParams* __restrict__ P, const double* __restrict__ F, const double* __restrict__ W,
              const double* __restrict__ sigma, const double* __restrict__ beta, double* At, double* Ab) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int S = P->S;
  if (i >= S) return;
  const double sg = sigma[i], bt = beta[i];
  At[i] = F[0 * S + i] + W[0 * S + i] * sg + W[1 * S + i] * bt;
  if (Ab) Ab[i] = F[1 * S + i] + W[1 * S + i] * sg + W[2 * S + i] * bt;
}

// Face state update of one Picard iteration: trial S_top (and fixed S_bot),
// residual and iterate norms from the constant weights, relaxation of sigma
// and beta, and the top reconstruction input of the relaxed iterate.
__global__ void __launch_bounds__(EW_THREADS)
k_fs_relax(const DevParams* __restrict__ P, const double* __restrict__ F, const double* __restrict__ W,
           const double* __restrict__ S_top, const double* __restrict__ S_bot, double* sigma, double* beta,
           double* At, double* partials) {
  __shared__ double sh[2 * (EW_THREADS / 32)];
  const int S = P->S;
  const double om = P->omega;
  double r2 = 0.0, o2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S; i += gridDim.x * blockDim.x) {
    const double sg = sigma[i], bt = beta[i];
    const double dt_ = S_top[i] - sg;
    const double db_ = (S_bot ? S_bot[i] : 0.0) - bt;
    const double qtt = W[3 * S + i], qtb = W[4 * S + i], qbb = W[5 * S + i];
    r2 += dt_ * dt_ * qtt + 2.0 * dt_ * db_ * qtb + db_ * db_ * qbb;
    o2 += 2.0 * (sg * F[2 * S + i] + bt * F[3 * S + i]) + sg * sg * qtt + 2.0 * sg * bt * qtb +
          bt * bt * qbb;
    const double ns = dt_ * om + sg;
    const double nb = db_ * om + bt;
    sigma[i] = ns;
    beta[i] = nb;
    At[i] = F[0 * S + i] + W[0 * S + i] * ns + W[1 * S + i] * nb;
  }
  block_sum2<EW_THREADS>(r2, o2, sh);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = r2;
    partials[2 * blockIdx.x + 1] = o2;
  }
}

// Commit of the modes: a = K a + KK (Ct sigma + Cb beta).
__global__ void __launch_bounds__(EW_THREADS)
k_fs_commit_modes(const DevParams* __restrict__ P, double* a, const double* __restrict__ K,
                  const double* __restrict__ KK, const double* __restrict__ Ct, const double* __restrict__ Cb,
                  const double* __restrict__ sigma, const double* __restrict__ beta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P->V) return;
  const int S = P->S;
  const int z = i / S, yx = i - z * S;
  const double kk = KK[i];
  a[i] = a[i] * K[i] + kk * (Ct[z] * sigma[yx] + Cb[z] * beta[yx]);
}

// Aligned sub-allocation of the caller's workspace.
struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
struct sgh_plan {
  sgh_config cfg;
  DevParams hp;
  int nparts_relax = 0, nparts_las = 0, nparts_surf = 0;
  int n_pre = 0, n_iter = 0, n_post = 0;  // kernels per step part (launch accounting)
  // offsets into the workspace
  size_t o_params, o_ctrl, o_mx, o_mxt, o_my, o_myt, o_mz, o_mzt, o_xc, o_yc, o_ct, o_cb;
  size_t o_K, o_KK, o_a, o_aK, o_trial, o_Tprev, o_Qm, o_t1, o_t2, o_vol, o_kp;
  size_t o_qlas, o_qnet, o_qev, o_qevold, o_Stop, o_Sbot, o_f1, o_f2, o_Tsurf, o_A;
  size_t o_prelax, o_plas, o_psurf, o_hist;
  int hist_cap = 0;
  // face-space Picard state: F (Zt, Zb, Yt, Yb), W (6 weights), sigma, beta, Ab, n1 partials
  bool face_space = false;
  int nparts_fs = 0, nparts_n1 = 0;
  size_t o_fsF = 0, o_fsW = 0, o_sigma = 0, o_beta = 0, o_Ab = 0, o_pn1 = 0;
  // box mode: point-major x/y tables, z reconstruction (+ face row) and
  // projection matrices, window bases, pass scratch, source and history
  double box_z0 = 0.0;
  size_t o_bx = 0, o_by = 0, o_bzi = 0, o_bzf = 0, o_wxi = 0, o_wxf = 0, o_wyi = 0, o_wyf = 0;
  size_t o_bt1 = 0, o_bt2 = 0, o_Qbox = 0, o_Tpb = 0, o_Qpb = 0, o_Tsh = 0, o_Qsh = 0;
  // mixed plans: BF16 pair planes of the transform and box matrices
  // (matrix offset, rows, contraction length, plane offset)
  struct PlaneSpec {
    size_t mat;
    int rows, k;
    size_t off;
    bool per_step;  // a window basis, rebuilt with the window every step
  };
  std::vector<PlaneSpec> plane_specs;
  std::vector<UmmaPlane> planes;
  bool bound_planes = false;
  size_t ws_need = 0;
  char* ws = nullptr;
  bool bound = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cs1 = nullptr, cs2 = nullptr;

  template <class T>
  T* at(size_t off) const { return reinterpret_cast<T*>(ws + off); }
  double* d(size_t off) const { return at<double>(off); }
  DevParams* P() const { return at<DevParams>(o_params); }
  Ctrl* ctrl() const { return at<Ctrl>(o_ctrl); }
};

namespace {

// Mixed-precision plan: every contraction on the split-BF16 tensor-core
// kernel, modal iterates rounded to FP32.
bool plan_mixed(const sgh_plan* p) { return p && p->cfg.precision == SGH_PRECISION_MIXED; }
// FP32 plan: every contraction in FP32 arithmetic on the CUDA cores, modal
// iterates rounded to FP32 (the FP32 arm of the precision study).
bool plan_fp32(const sgh_plan* p) { return p && p->cfg.precision == SGH_PRECISION_FP32; }
int* umma_err_of(const sgh_plan* p) { return (p && p->ws) ? &p->ctrl()->umma_err : nullptr; }
// The plan's matrices with BF16 pair planes (mixed plans, once bound).
const UmmaPlane* planes_of(const sgh_plan* p) { return (p && p->bound_planes) ? p->planes.data() : nullptr; }
int nplanes_of(const sgh_plan* p) { return (p && p->bound_planes) ? (int)p->planes.size() : 0; }

int check_program(const sgh_program& p, const char* name) {
  if (p.n_ops < 1 || p.n_ops > SGH_MAX_PROGRAM || p.n_consts < 0 || p.n_consts > SGH_MAX_CONSTS)
    return fail(SGH_ERR_INVALID, std::string("property program ") + name + " has a bad size");
  int depth = 0;
  for (int i = 0; i < p.n_ops;) {
    const int op = p.ops[i++];
    if (op == SGH_OP_CONST) {
      if (i >= p.n_ops || p.ops[i] < 0 || p.ops[i] >= p.n_consts)
        return fail(SGH_ERR_INVALID, std::string("property program ") + name + " has a bad constant");
      ++i;
      ++depth;
    } else if (op == SGH_OP_T) {
      ++depth;
    } else if ((op >= SGH_OP_ADD && op <= SGH_OP_POW) || op == SGH_OP_ATAN2) {
      if (depth < 2) return fail(SGH_ERR_INVALID, std::string("property program ") + name + " underflows");
      --depth;
    } else if (op == SGH_OP_NEG || (op >= SGH_OP_SQRT && op <= SGH_OP_EXPM1)) {
      if (depth < 1) return fail(SGH_ERR_INVALID, std::string("property program ") + name + " underflows");
    } else {
      return fail(SGH_ERR_INVALID, std::string("property program ") + name + " has an unknown opcode");
    }
    if (depth > SGH_MAX_STACK) return fail(SGH_ERR_INVALID, std::string("property program ") + name + " is too deep");
  }
  if (depth != 1) return fail(SGH_ERR_INVALID, std::string("property program ") + name + " leaves a bad stack");
  return SGH_OK;
}

// Abstract interpretation of a property program over affine forms a + b T:
// true (with the coefficients) when the program is affine in T, as the
// piecewise-linear property tables are; constants are folded with host libm.
bool program_affine(const sgh_program& p, double* A, double* B) {
  double sa[SGH_MAX_STACK + 1], sb[SGH_MAX_STACK + 1];
  int sp = 0;
  for (int i = 0; i < p.n_ops;) {
    const int op = p.ops[i++];
    if (op == SGH_OP_CONST) { sa[sp] = p.consts[p.ops[i++]]; sb[sp] = 0.0; ++sp; continue; }
    if (op == SGH_OP_T) { sa[sp] = 0.0; sb[sp] = 1.0; ++sp; continue; }
    if ((op >= SGH_OP_ADD && op <= SGH_OP_POW) || op == SGH_OP_ATAN2) {
      --sp;
      const double xa = sa[sp - 1], xb = sb[sp - 1], ya = sa[sp], yb = sb[sp];
      double ra, rb;
      switch (op) {
        case SGH_OP_ADD: ra = xa + ya; rb = xb + yb; break;
        case SGH_OP_SUB: ra = xa - ya; rb = xb - yb; break;
        case SGH_OP_MUL:
          if (xb == 0.0) { ra = xa * ya; rb = xa * yb; }
          else if (yb == 0.0) { ra = xa * ya; rb = xb * ya; }
          else return false;
          break;
        case SGH_OP_DIV:
          if (yb != 0.0) return false;
          ra = xa / ya; rb = xb / ya;
          break;
        case SGH_OP_POW:
          if (xb != 0.0 || yb != 0.0) return false;
          ra = std::pow(xa, ya); rb = 0.0;
          break;
        default:  // atan2
          if (xb != 0.0 || yb != 0.0) return false;
          ra = std::atan2(xa, ya); rb = 0.0;
      }
      sa[sp - 1] = ra; sb[sp - 1] = rb;
      continue;
    }
    if (op == SGH_OP_NEG) { sa[sp - 1] = -sa[sp - 1]; sb[sp - 1] = -sb[sp - 1]; continue; }
    if (sb[sp - 1] != 0.0) return false;  // a function of T: not affine
    const double x = sa[sp - 1];
    double r;
    switch (op) {
      case SGH_OP_SQRT: r = std::sqrt(x); break;
      case SGH_OP_EXP: r = std::exp(x); break;
      case SGH_OP_LOG: r = std::log(x); break;
      case SGH_OP_LOG2: r = std::log2(x); break;
      case SGH_OP_LOG10: r = std::log10(x); break;
      case SGH_OP_SIN: r = std::sin(x); break;
      case SGH_OP_COS: r = std::cos(x); break;
      case SGH_OP_TAN: r = std::tan(x); break;
      case SGH_OP_ASIN: r = std::asin(x); break;
      case SGH_OP_ACOS: r = std::acos(x); break;
      case SGH_OP_ATAN: r = std::atan(x); break;
      case SGH_OP_SINH: r = std::sinh(x); break;
      case SGH_OP_COSH: r = std::cosh(x); break;
      case SGH_OP_TANH: r = std::tanh(x); break;
      case SGH_OP_ASINH: r = std::asinh(x); break;
      case SGH_OP_ACOSH: r = std::acosh(x); break;
      case SGH_OP_ATANH: r = std::atanh(x); break;
      case SGH_OP_FABS: r = std::fabs(x); break;
      case SGH_OP_CEIL: r = std::ceil(x); break;
      case SGH_OP_FLOOR: r = std::floor(x); break;
      case SGH_OP_TRUNC: r = std::trunc(x); break;
      case SGH_OP_LOG1P: r = std::log1p(x); break;
      case SGH_OP_EXPM1: r = std::expm1(x); break;
      default: return false;
    }
    sa[sp - 1] = r;
  }
  if (sp != 1) return false;
  *A = sa[0];
  *B = sb[0];
  return std::isfinite(*A) && std::isfinite(*B);
}

// ---- enqueue helpers (used both for graph capture and for direct calls) ----

template <class Epi>
inline void axis(const double* X, const double* Mat, int Nout, int N, int A, int B, const Epi& epi,
                 cudaStream_t st) {
  launch_axis(X, Mat, Nout, N, A, B, epi, st);
  ++g_launches;
}

template <class Epi>
void face_dct2_epi(sgh_plan* p, const double* in, const Epi& epi, cudaStream_t s) {
  const DevParams& h = p->hp;
  axis(in, p->d(p->o_mx), h.nx, h.nx, h.ny, 1, EpiStore{p->d(p->o_f1), 1.0, nullptr}, s);
  axis(p->d(p->o_f1), p->d(p->o_my), h.ny, h.ny, 1, h.nx, epi, s);
}

void face_dct2(sgh_plan* p, const double* in, double* out, double scale, cudaStream_t s) {
  face_dct2_epi(p, in, EpiStore{out, scale, nullptr}, s);
}

// Face IDCT2 of a prepared face input A (no z-sum).
template <class Epi>
void face_idct2_from(sgh_plan* p, const double* A, const Epi& epi, cudaStream_t s) {
  const DevParams& h = p->hp;
  axis(A, p->d(p->o_mxt), h.nx, h.nx, h.ny, 1, EpiStore{p->d(p->o_f1), 1.0, nullptr}, s);
  axis(p->d(p->o_f1), p->d(p->o_myt), h.ny, h.ny, 1, h.nx, epi, s);
}

template <class Epi>
void face_idct2(sgh_plan* p, const double* modes, const double* w, const Epi& epi, cudaStream_t s) {
  const DevParams& h = p->hp;
  k_zsum<<<cdiv(h.S, EW_THREADS), EW_THREADS, 0, s>>>(modes, w, h.nz, h.S, p->d(p->o_A));
  ++g_launches;
  axis(p->d(p->o_A), p->d(p->o_mxt), h.nx, h.nx, h.ny, 1, EpiStore{p->d(p->o_f1), 1.0, nullptr}, s);
  axis(p->d(p->o_f1), p->d(p->o_myt), h.ny, h.ny, 1, h.nx, epi, s);
}

// Three passes x -> y -> z through t1, t2; the last pass applies epi.
// slabs: z-slabs run through the x and y passes (nz, or nz + 1 when the
// input carries a face field as slab nz); z_rows: output rows of the z-pass
// (nz, or nz + 1 / nz + 2 for the inverse with the surface rows appended).
template <class Epi>
void volume_pass3(sgh_plan* p, const double* in, bool inverse, const Epi& epi, double* t1, double* t2,
                  cudaStream_t s, int slabs = -1, int z_rows = -1) {
  const DevParams& h = p->hp;
  if (slabs < 0) slabs = h.nz;
  if (z_rows < 0) z_rows = h.nz;
  const double* mx = p->d(inverse ? p->o_mxt : p->o_mx);
  const double* my = p->d(inverse ? p->o_myt : p->o_my);
  const double* mz = p->d(inverse ? p->o_mzt : p->o_mz);
  axis(in, mx, h.nx, h.nx, h.ny * slabs, 1, EpiStore{t1, 1.0, nullptr}, s);
  axis(t1, my, h.ny, h.ny, slabs, h.nx, EpiStore{t2, 1.0, nullptr}, s);
  axis(t2, mz, z_rows, h.nz, 1, h.S, epi, s);
}

// ---- box passes (order z, x, y for a reconstruction; y, x, z for a projection:
// the contraction order of least work when the box is shallow in z) ----

// z-pass of a box reconstruction of modes into bt1: rows 0..zb-1 of the box
// bases, and with the face row (the top weights Ct) the z-summed input of the
// top-surface temperature as slab zb (einsum 'p,pij->ij', spectral_ops.py:210-219).
void box_zpass(sgh_plan* p, const double* modes, bool with_face, cudaStream_t s) {
  const DevParams& h = p->hp;
  axis(modes, p->d(p->o_bzi), h.zb + (with_face ? 1 : 0), h.nz, 1, h.S,
       EpiStore{p->d(p->o_bt1), 1.0, nullptr}, s);
}

// x- and y-passes of a box reconstruction from bt1; epi receives T_box.
template <class Epi>
void box_xy(sgh_plan* p, const Epi& epi, cudaStream_t s) {
  const DevParams& h = p->hp;
  axis(p->d(p->o_bt1), p->d(p->o_wxi), h.xb, h.nx, h.zb * h.ny, 1, EpiStore{p->d(p->o_bt2), 1.0, nullptr}, s);
  axis(p->d(p->o_bt2), p->d(p->o_wyi), h.yb, h.ny, h.zb, h.xb, epi, s);
}

// Projection of a box field onto the modes (project_box_to_modes,
// physics/spectral_ops.py:53-74); epi receives the contraction before the
// dV_fine scale.
template <class Epi>
void box_project(sgh_plan* p, const double* field, const Epi& epi, cudaStream_t s) {
  const DevParams& h = p->hp;
  axis(field, p->d(p->o_wyf), h.ny, h.yb, h.zb, h.xb, EpiStore{p->d(p->o_bt2), 1.0, nullptr}, s);
  axis(p->d(p->o_bt2), p->d(p->o_wxf), h.nx, h.xb, h.zb * h.ny, 1, EpiStore{p->d(p->o_bt1), 1.0, nullptr}, s);
  axis(p->d(p->o_bt1), p->d(p->o_bzf), h.nz, h.zb, 1, h.S, epi, s);
}

// First step of a run: seed T_prev = T_box(aK) and Q_prev = 0
// (initialize_latent_heat_if_needed, physics/spectral_ops.py:182-194). Every
// launch is guarded by the history flag, so eager calls may enqueue it each
// step; the graph runs it under a conditional node.
void enqueue_box_seed(sgh_plan* p, cudaStream_t s) {
  const DevParams& h = p->hp;
  k_box_seed<<<cdiv(h.V, EW_THREADS), EW_THREADS, 0, s>>>(p->P(), p->ctrl(), p->d(p->o_a), p->d(p->o_K),
                                                          p->d(p->o_aK));
  ++g_launches;
  box_zpass(p, p->d(p->o_aK), false, s);
  box_xy(p, EpiBoxInit{p->ctrl(), p->d(p->o_Tpb), p->d(p->o_Qpb), nullptr}, s);
}

void enqueue_pre_face_space(sgh_plan* p, cudaStream_t s) {
  const DevParams& h = p->hp;
  DevParams* P = p->P();
  const PointPhys PP = point_phys(p->hp, P);
  const int gS = cdiv(h.S, EW_THREADS);
  double* F = p->d(p->o_fsF);
  double* W = p->d(p->o_fsW);
  double* sg = p->d(p->o_sigma);
  double* bt = p->d(p->o_beta);
  double* At = p->d(p->o_A);
  double* Ab = p->d(p->o_Ab);
  k_fs_pass1<<<gS, EW_THREADS, 0, s>>>(P, p->d(p->o_a), p->d(p->o_K), p->d(p->o_KK), p->d(p->o_ct),
                                        p->d(p->o_cb), F, p->d(p->o_pn1));
  ++g_launches;
  SGH_CK_VOID(cudaMemsetAsync(bt, 0, sizeof(double) * h.S, s));
  face_dct2(p, p->d(p->o_qnet), sg, h.dct_scale, s);  // initial guess sigma = S_top
  if (h.has_top_conv) {
    k_fs_assemble<<<gS, EW_THREADS, 0, s>>>(P, F, W, sg, bt, At, nullptr);
    ++g_launches;
    face_idct2_from(p, At, EpiConvFace{PP, h.h_top, 0, p->d(p->o_f2), nullptr}, s);
    face_dct2_epi(p, p->d(p->o_f2), EpiAdd{sg, h.dct_scale, nullptr}, s);
  }
  if (h.has_bottom_conv) {
    k_fs_assemble<<<gS, EW_THREADS, 0, s>>>(P, F, W, sg, bt, At, Ab);
    ++g_launches;
    face_idct2_from(p, Ab, EpiConvFace{PP, h.h_bottom, 0, p->d(p->o_f2), nullptr}, s);
    face_dct2_epi(p, p->d(p->o_f2), EpiAdd{bt, h.dct_scale, nullptr}, s);
    // S_bot_raw, held fixed through the Picard loop (solvers/spectral.py:373-379)
    k_fs_assemble<<<gS, EW_THREADS, 0, s>>>(P, F, W, sg, bt, At, Ab);
    ++g_launches;
    face_idct2_from(p, Ab, EpiConvFace{PP, h.h_bottom, 0, p->d(p->o_f2), nullptr}, s);
    face_dct2(p, p->d(p->o_f2), p->d(p->o_Sbot), h.dct_scale, s);
  }
  k_fs_assemble<<<gS, EW_THREADS, 0, s>>>(P, F, W, sg, bt, At, nullptr);
  ++g_launches;
}

void enqueue_picard_face_space(sgh_plan* p, cudaStream_t s, cudaGraphConditionalHandle h_picard,
                               int in_graph) {
  const DevParams& h = p->hp;
  DevParams* P = p->P();
  const PointPhys PP = point_phys(p->hp, P);
  face_idct2_from(p, p->d(p->o_A),
                  EpiTopFlux{PP, p->d(p->o_qlas), p->d(p->o_qev), p->d(p->o_qnet), 0, nullptr}, s);
  face_dct2(p, p->d(p->o_qnet), p->d(p->o_Stop), h.dct_scale, s);
  k_fs_relax<<<p->nparts_fs, EW_THREADS, 0, s>>>(P, p->d(p->o_fsF), p->d(p->o_fsW), p->d(p->o_Stop),
                                                 h.has_bottom_conv ? p->d(p->o_Sbot) : nullptr,
                                                 p->d(p->o_sigma), p->d(p->o_beta), p->d(p->o_A),
                                                 p->d(p->o_prelax));
  ++g_launches;
  k_converge<<<1, EW_THREADS, 0, s>>>(P, p->ctrl(), p->d(p->o_prelax), p->nparts_fs, p->d(p->o_pn1),
                                       p->nparts_n1, h_picard, in_graph);
  ++g_launches;
}

// BF16 pair plane of one matrix of a mixed plan.
void build_plane(sgh_plan* p, const sgh_plan::PlaneSpec& q, cudaStream_t s) {
  const long n = (long)cdiv(q.rows, AXU_M) * AXU_M * (long)cdiv(q.k, AXU_KC) * AXU_KC;
  k_pair_plane<<<std::min(cdiv(n, EW_THREADS), 1184), EW_THREADS, 0, s>>>(p->d(q.mat), q.rows, q.k, p->ws + q.off);
}

// Step opening: laser state, Picard switch, face forcing and (box mode) the
// window of this step.
void enqueue_pre_begin(sgh_plan* p, cudaStream_t s, cudaGraphConditionalHandle h_picard,
                       cudaGraphConditionalHandle h_seed, int in_graph) {
  const DevParams& h = p->hp;
  DevParams* P = p->P();
  const PointPhys PP = point_phys(p->hp, P);
  Ctrl* C = p->ctrl();
  const int gS = cdiv(h.S, EW_THREADS);
  k_step_begin<<<1, 1, 0, s>>>(P, C, h_picard, h_seed, in_graph);
  ++g_launches;
  k_face_begin<<<gS, EW_THREADS, 0, s>>>(P, C, p->d(p->o_xc), p->d(p->o_yc), p->d(p->o_qevold),
                                          p->d(p->o_qlas), p->d(p->o_qnet), p->d(p->o_plas));
  ++g_launches;
  if (h.box) {
    const long long n = (long long)h.xb * h.nx + (long long)h.yb * h.ny;
    k_box_window<<<cdiv(n, EW_THREADS), EW_THREADS, 0, s>>>(P, C, p->d(p->o_bx), p->d(p->o_by), p->d(p->o_wxi),
                                                            p->d(p->o_wxf), p->d(p->o_wyi), p->d(p->o_wyf));
    ++g_launches;
    for (const auto& q : p->plane_specs)
      if (q.per_step) {
        build_plane(p, q, s);
        ++g_launches;
      }
  }
}

// Rest of the step opening: (box mode) history shift and its projection,
// initial guess and the convection guesses.
void enqueue_pre_rest(sgh_plan* p, cudaStream_t s) {
  const DevParams& h = p->hp;
  DevParams* P = p->P();
  const PointPhys PP = point_phys(p->hp, P);
  Ctrl* C = p->ctrl();
  const int gV = cdiv(h.V, EW_THREADS);
  if (p->face_space) {
    enqueue_pre_face_space(p, s);
    return;
  }
  if (h.box) {
    k_box_shift<<<cdiv(h.Nb, EW_THREADS), EW_THREADS, 0, s>>>(P, C, p->d(p->o_Tpb), p->d(p->o_Qpb),
                                                              p->d(p->o_Tsh), p->d(p->o_Qsh));
    ++g_launches;
    // warm start: the shifted source of the previous step, projected (solvers/spectral.py:323-327)
    box_project(p, p->d(p->o_Qsh), EpiStore{p->d(p->o_Qm), h.dV_fine, nullptr}, s);
  }
  face_dct2(p, p->d(p->o_qnet), p->d(p->o_Stop), h.dct_scale, s);
  k_init_modes<<<gV, EW_THREADS, 0, s>>>(P, C, p->d(p->o_a), p->d(p->o_K), p->d(p->o_KK), p->d(p->o_ct),
                                          p->d(p->o_Stop), p->d(p->o_Qm), p->d(p->o_aK));
  ++g_launches;
  if (h.has_top_conv) {
    face_idct2(p, p->d(p->o_a), p->d(p->o_ct), EpiConvFace{PP, h.h_top, 0, p->d(p->o_f2), nullptr}, s);
    face_dct2(p, p->d(p->o_f2), p->d(p->o_Stop), h.dct_scale, s);
    k_add_face<<<gV, EW_THREADS, 0, s>>>(P, p->d(p->o_a), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_Stop));
  ++g_launches;
  }
  if (h.has_bottom_conv) {
    face_idct2(p, p->d(p->o_a), p->d(p->o_cb), EpiConvFace{PP, h.h_bottom, 0, p->d(p->o_f2), nullptr}, s);
    face_dct2(p, p->d(p->o_f2), p->d(p->o_Sbot), h.dct_scale, s);
    k_add_face<<<gV, EW_THREADS, 0, s>>>(P, p->d(p->o_a), p->d(p->o_KK), p->d(p->o_cb), p->d(p->o_Sbot));
  ++g_launches;
    // S_bot_raw, held fixed through the Picard loop (solvers/spectral.py:373-379)
    face_idct2(p, p->d(p->o_a), p->d(p->o_cb),
               EpiConvFace{PP, h.h_bottom, h.prop_corr, p->d(p->o_f2), nullptr}, s);
    face_dct2(p, p->d(p->o_f2), p->d(p->o_Sbot), h.dct_scale, s);
  }
}

void enqueue_pre(sgh_plan* p, cudaStream_t s) {
  enqueue_pre_begin(p, s, 0, 0, 0);
  if (p->hp.box) enqueue_box_seed(p, s);
  enqueue_pre_rest(p, s);
}

void enqueue_picard(sgh_plan* p, cudaStream_t s, cudaGraphConditionalHandle h_picard, int in_graph) {
  if (p->face_space) {
    enqueue_picard_face_space(p, s, h_picard, in_graph);
    return;
  }
  const DevParams& h = p->hp;
  DevParams* P = p->P();
  const PointPhys PP = point_phys(p->hp, P);
  Ctrl* C = p->ctrl();
  const int gV = cdiv(h.V, EW_THREADS);
  double* S_bot = h.has_bottom_conv ? p->d(p->o_Sbot) : nullptr;
  int nparts = 0;
  if (h.box) {
    // box z-pass with the face row, top flux from the face row, the latent
    // source on the box, and its projection into the trial modes
    // (solvers/spectral.py:388-443 with the box branch :413-422)
    box_zpass(p, p->d(p->o_a), true, s);
    face_idct2_from(p, p->d(p->o_bt1) + (size_t)h.zb * h.S,
                    EpiTopFlux{PP, p->d(p->o_qlas), p->d(p->o_qev), p->d(p->o_qnet), h.prop_corr, nullptr}, s);
    face_dct2(p, p->d(p->o_qnet), p->d(p->o_Stop), h.dct_scale, s);
    box_xy(p, EpiBoxLatent{PP, p->d(p->o_Tsh), p->d(p->o_Qbox), nullptr, h.latent_model, h.T_solidus, h.band_inv,
                           h.latent_factor},
           s);
    if (h.prop_corr) {
      box_project(p, p->d(p->o_Qbox),
                  EpiTrial<false>{PP, p->d(p->o_aK), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb), p->d(p->o_Stop),
                                  1.0, h.dV_fine, S_bot, nullptr, p->d(p->o_trial), nullptr, nullptr, h.S, h.omega},
                  s);
    } else {
      box_project(p, p->d(p->o_Qbox),
                  EpiTrial<true>{PP, p->d(p->o_aK), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb), p->d(p->o_Stop),
                                 1.0, h.dV_fine, S_bot, nullptr, nullptr, p->d(p->o_a), p->d(p->o_prelax), h.S,
                                 h.omega},
                  s);
      nparts = axis_blocks(h.nz, 1, h.S);
    }
  } else if (h.grid_latent) {
    // IDCT3(a_old) with the surface row: latent source in slabs 0..nz-1 and
    // the net top flux in slab nz of vol; then DCT3 over nz + 1 slabs turns
    // slab nz into DCT2(q_net), read by the trial epilogue as S_top.
    volume_pass3(p, p->d(p->o_a), true,
                 EpiLatentSurface{PP, p->d(p->o_Tprev), p->d(p->o_vol), p->d(p->o_qlas), p->d(p->o_qev),
                                  h.prop_corr, nullptr},
                 p->d(p->o_t1), p->d(p->o_t2), s, h.nz, h.nz + 1);
    const double* S_top = p->d(p->o_t2) + (size_t)h.nz * h.S;
    if (h.prop_corr) {
      volume_pass3(p, p->d(p->o_vol), false,
                   EpiTrial<false>{PP, p->d(p->o_aK), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb),
                                   S_top, h.dct_scale, h.sqrt_dV, S_bot, p->d(p->o_Qm), p->d(p->o_trial),
                                   nullptr, nullptr, h.S, h.omega},
                   p->d(p->o_t1), p->d(p->o_t2), s, h.nz + 1, h.nz);
    } else {
      volume_pass3(p, p->d(p->o_vol), false,
                   EpiTrial<true>{PP, p->d(p->o_aK), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb),
                                  S_top, h.dct_scale, h.sqrt_dV, S_bot, p->d(p->o_Qm), nullptr, p->d(p->o_a),
                                  p->d(p->o_prelax), h.S, h.omega},
                   p->d(p->o_t1), p->d(p->o_t2), s, h.nz + 1, h.nz);
      nparts = axis_blocks(h.nz, 1, h.S);
    }
  } else {
    // top face: T_s, evaporation, convection, rescale -> S_top
    face_idct2(p, p->d(p->o_a), p->d(p->o_ct),
               EpiTopFlux{PP, p->d(p->o_qlas), p->d(p->o_qev), p->d(p->o_qnet), h.prop_corr, nullptr}, s);
    face_dct2(p, p->d(p->o_qnet), p->d(p->o_Stop), h.dct_scale, s);
  }
  if (!h.grid_latent && !h.box && h.prop_corr) {
    k_trial<<<gV, EW_THREADS, 0, s>>>(P, p->d(p->o_aK), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb),
                                       p->d(p->o_Stop), S_bot, p->d(p->o_trial));
    ++g_launches;
  } else if (!h.grid_latent && !h.box) {
    const int g = p->nparts_relax;
    k_trial_relax<<<g, EW_THREADS, 0, s>>>(P, p->d(p->o_aK), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb),
                                            p->d(p->o_Stop), S_bot, p->d(p->o_a), p->d(p->o_prelax));
    ++g_launches;
    nparts = g;
  }
  if (h.prop_corr) {
    volume_pass3(p, p->d(p->o_trial), true,
                 EpiTemperatureKp{PP, p->d(p->o_vol), p->d(p->o_kp), nullptr}, p->d(p->o_t1),
                 p->d(p->o_t2), s);
    k_stencil<<<gV, EW_THREADS, 0, s>>>(P, p->d(p->o_vol), p->d(p->o_kp), p->d(p->o_Tprev), p->d(p->o_t1));
    ++g_launches;
    volume_pass3(p, p->d(p->o_t1), false,
                 EpiRelax{PP, p->d(p->o_trial), p->d(p->o_KK), p->d(p->o_a), p->d(p->o_prelax)},
                 p->d(p->o_t2), p->d(p->o_vol), s);
    nparts = axis_blocks(h.nz, 1, h.S);
  }
  k_converge<<<1, EW_THREADS, 0, s>>>(P, C, p->d(p->o_prelax), nparts, nullptr, 0, h_picard, in_graph);
  ++g_launches;
}

void enqueue_post(sgh_plan* p, cudaStream_t s, cudaGraphConditionalHandle h_steps, int in_graph) {
  const DevParams& h = p->hp;
  DevParams* P = p->P();
  const PointPhys PP = point_phys(p->hp, P);
  int n_surf;
  if (h.box) {
    // surface of the committed modes (from the box z-pass face row unless the
    // property correction commits the full volume), then the box history:
    // T_prev = T_box(a), Q_prev = the last source (solvers/spectral.py:502-533)
    if (h.prop_corr) {
      volume_pass3(p, p->d(p->o_a), true,
                   EpiCommitVolume{PP, p->d(p->o_Tprev), p->d(p->o_Tsurf), p->d(p->o_qev), p->d(p->o_qevold),
                                   p->d(p->o_psurf)},
                   p->d(p->o_t1), p->d(p->o_t2), s, h.nz, h.nz + 1);
      n_surf = axis_blocks(h.nz + 1, 1, h.S);
      box_zpass(p, p->d(p->o_a), false, s);
    } else {
      box_zpass(p, p->d(p->o_a), true, s);
      face_idct2_from(p, p->d(p->o_bt1) + (size_t)h.zb * h.S,
                      EpiCommitSurface{PP, p->d(p->o_Tsurf), p->d(p->o_qev), p->d(p->o_qevold), p->d(p->o_psurf)},
                      s);
      n_surf = p->nparts_surf;
    }
    box_xy(p, EpiBoxCommit{p->ctrl(), p->d(p->o_Tpb), p->d(p->o_Qpb), p->d(p->o_Qbox), p->d(p->o_Qsh), nullptr}, s);
    k_box_check<<<std::min(4 * 148, cdiv(h.Nb, EW_THREADS)), EW_THREADS, 0, s>>>(P, p->ctrl(), p->d(p->o_Qpb));
    ++g_launches;
  } else if (p->face_space) {
    face_idct2_from(p, p->d(p->o_A),
                    EpiCommitSurface{PP, p->d(p->o_Tsurf), p->d(p->o_qev), p->d(p->o_qevold), p->d(p->o_psurf)},
                    s);
    k_fs_commit_modes<<<cdiv(h.V, EW_THREADS), EW_THREADS, 0, s>>>(
        P, p->d(p->o_a), p->d(p->o_K), p->d(p->o_KK), p->d(p->o_ct), p->d(p->o_cb), p->d(p->o_sigma),
        p->d(p->o_beta));
    ++g_launches;
    n_surf = p->nparts_surf;
  } else if (h.grid_latent || h.prop_corr) {
    // T_prev and the surface temperature from one IDCT3 with the surface row
    volume_pass3(p, p->d(p->o_a), true,
                 EpiCommitVolume{PP, p->d(p->o_Tprev), p->d(p->o_Tsurf), p->d(p->o_qev), p->d(p->o_qevold),
                                 p->d(p->o_psurf)},
                 p->d(p->o_t1), p->d(p->o_t2), s, h.nz, h.nz + 1);
    n_surf = axis_blocks(h.nz + 1, 1, h.S);
  } else {
    face_idct2(p, p->d(p->o_a), p->d(p->o_ct),
               EpiCommitSurface{PP, p->d(p->o_Tsurf), p->d(p->o_qev), p->d(p->o_qevold), p->d(p->o_psurf)}, s);
    n_surf = p->nparts_surf;
  }
  k_commit<<<1, EW_THREADS, 0, s>>>(P, p->ctrl(), p->d(p->o_plas), p->nparts_las, p->d(p->o_psurf),
                                     n_surf, h_steps, in_graph);
  ++g_launches;
}

// Adds a conditional node of the given type to the graph being captured on
// cs (after the captured work so far) and returns its body graph.
int add_conditional(cudaStream_t cs, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body) {
  cudaStreamCaptureStatus status;
  cudaGraph_t cur;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  SGH_CK(cudaStreamGetCaptureInfo(cs, &status, nullptr, &cur, &deps, &ndeps));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  SGH_CK(cudaGraphAddNode(&node, cur, deps, ndeps, &np));
  SGH_CK(cudaStreamUpdateCaptureDependencies(cs, &node, 1, cudaStreamSetCaptureDependencies));
  *body = np.conditional.phGraph_out[0];
  return SGH_OK;
}

int capture(sgh_plan* p) {
  cudaGraph_t G;
  SGH_CK(cudaGraphCreate(&G, 0));
  p->graph = G;
  cudaGraphConditionalHandle h_steps;
  SGH_CK(cudaGraphConditionalHandleCreate(&h_steps, G, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams outer = {};
  outer.type = cudaGraphNodeTypeConditional;
  outer.conditional.handle = h_steps;
  outer.conditional.type = cudaGraphCondTypeWhile;
  outer.conditional.size = 1;
  cudaGraphNode_t outer_node;
  SGH_CK(cudaGraphAddNode(&outer_node, G, nullptr, 0, &outer));
  cudaGraph_t body = outer.conditional.phGraph_out[0];

  SGH_CK(cudaStreamBeginCaptureToGraph(p->cs1, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cudaGraphConditionalHandle h_picard, h_seed = 0;
  SGH_CK(cudaGraphConditionalHandleCreate(&h_picard, body, 0, 0));
  if (p->hp.box) SGH_CK(cudaGraphConditionalHandleCreate(&h_seed, body, 0, 0));
  g_launches = 0;
  enqueue_pre_begin(p, p->cs1, h_picard, h_seed, 1);
  if (p->hp.box) {
    // history seeding, first step of a run only (not counted per step)
    cudaGraph_t sbody;
    const int rc = add_conditional(p->cs1, h_seed, cudaGraphCondTypeIf, &sbody);
    if (rc) return rc;
    const int saved = g_launches;
    SGH_CK(cudaStreamBeginCaptureToGraph(p->cs2, sbody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_box_seed(p, p->cs2);
    SGH_CK(cudaStreamEndCapture(p->cs2, &sbody));
    g_launches = saved;
  }
  enqueue_pre_rest(p, p->cs1);
  p->n_pre = g_launches;
  cudaGraph_t ibody;
  {
    const int rc = add_conditional(p->cs1, h_picard, cudaGraphCondTypeWhile, &ibody);
    if (rc) return rc;
  }
  SGH_CK(cudaStreamBeginCaptureToGraph(p->cs2, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  g_launches = 0;
  enqueue_picard(p, p->cs2, h_picard, 1);
  p->n_iter = g_launches;
  SGH_CK(cudaStreamEndCapture(p->cs2, &ibody));
  g_launches = 0;
  enqueue_post(p, p->cs1, h_steps, 1);
  p->n_post = g_launches;
  SGH_CK(cudaStreamEndCapture(p->cs1, &body));
  SGH_CK(cudaGetLastError());
  SGH_CK(cudaGraphInstantiate(&p->exec, G, 0));
  return SGH_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int sgh_abi_version(void) { return SGH_ABI_VERSION; }

const char* sgh_last_error(void) { return g_last_error.c_str(); }

int sgh_plan_create(const sgh_config* cfg, sgh_plan** out) {
  if (!cfg || !out) return fail(SGH_ERR_INVALID, "null argument");
  *out = nullptr;
  const sgh_config& c = *cfg;
  if (c.axis_min_ctas < 0) return fail(SGH_ERR_INVALID, "axis_min_ctas must be >= 0");
  if (c.axis_cuda_cores != 0 && c.axis_cuda_cores != 1) return fail(SGH_ERR_INVALID, "axis_cuda_cores must be 0 or 1");
  AxisPolicy policy(c.axis_min_ctas, c.axis_cuda_cores, c.precision == SGH_PRECISION_MIXED, nullptr,
                    c.precision == SGH_PRECISION_FP32);
  if (c.nx < 2 || c.ny < 2 || c.nz < 2) return fail(SGH_ERR_INVALID, "every axis needs at least 2 modes");
  if (c.nx > 4096 || c.ny > 4096 || c.nz > 4096) return fail(SGH_ERR_INVALID, "an axis exceeds 4096 modes");
  if ((long long)c.nx * c.ny * c.nz > (1LL << 28)) return fail(SGH_ERR_INVALID, "grid exceeds 2^28 modes");
  if (c.precision != SGH_PRECISION_FP64 && c.precision != SGH_PRECISION_MIXED &&
      c.precision != SGH_PRECISION_FP32)
    return fail(SGH_ERR_INVALID, "precision must be SGH_PRECISION_FP64, _MIXED or _FP32");
  if (!(c.Lx > 0 && c.Ly > 0 && c.Lz > 0 && c.dt > 0))
    return fail(SGH_ERR_INVALID, "domain size and dt must be positive");
  if (!(c.r_x > 0 && c.r_y > 0 && c.area_factor > 0 && c.order > 0))
    return fail(SGH_ERR_INVALID, "beam radii, order and area factor must be positive");
  if (c.max_iter < 0 || c.max_iter > 1000000)
    return fail(SGH_ERR_INVALID, "max_iter must be in [0, 1e6]");
  if (c.cell_integrated && c.order != 2.0)
    return fail(SGH_ERR_INVALID, "cell_integrated flux is only defined for the Gaussian (order 2)");
  const bool prop_corr = c.has_model && !c.model_constant;
  const bool latent = c.L_f > 0.0;
  const bool box = c.box != 0;
  if (latent && !(c.has_model && !c.model_constant) && !(c.T_liquidus > c.T_solidus))
    return fail(SGH_ERR_INVALID, "latent heat with constant properties needs T_liquidus > T_solidus");
  if (box) {
    if (c.box_refinement < 1 || c.box_refinement > 64)
      return fail(SGH_ERR_INVALID, "box_refinement must be in [1, 64]");
    if (!(c.box_size[0] > 0 && c.box_size[1] > 0 && c.box_size[2] > 0))
      return fail(SGH_ERR_INVALID, "box_size must be positive");
    if (!prop_corr && !(c.T_liquidus > c.T_solidus))
      return fail(SGH_ERR_INVALID, "box mode with constant properties needs T_liquidus > T_solidus");
  }
  if (c.has_model) {
    const sgh_program* progs[6] = {&c.k_solid, &c.k_liquid, &c.rho_solid, &c.rho_liquid, &c.c_solid, &c.c_liquid};
    const char* names[6] = {"k_solid", "k_liquid", "rho_solid", "rho_liquid", "c_solid", "c_liquid"};
    for (int i = 0; i < 6; ++i) {
      const int rc = check_program(*progs[i], names[i]);
      if (rc) return rc;
    }
  }

  sgh_plan* p = new sgh_plan();
  p->cfg = c;
  DevParams& h = p->hp;
  std::memset(&h, 0, sizeof(h));
  h.round32 = c.precision != SGH_PRECISION_FP64 ? 1 : 0;
  h.nx = c.nx; h.ny = c.ny; h.nz = c.nz;
  h.S = c.nx * c.ny;
  h.V = h.S * c.nz;
  h.grid_latent = latent && !box;  // grid mode: no fine box (solvers/spectral.py:182-186)
  h.box = box;
  h.prop_corr = prop_corr;
  h.latent_model = prop_corr;  // blended-rho source only for a non-constant model
  h.k_constant = c.k_constant;
  h.has_top_conv = c.h_top > 0.0;
  h.has_bottom_conv = c.h_bottom > 0.0;
  h.cell_integrated = c.cell_integrated;
  h.max_iter = c.max_iter;
  h.Lx = c.Lx; h.Ly = c.Ly; h.Lz = c.Lz;
  h.dx = c.Lx / c.nx; h.dy = c.Ly / c.ny; h.dz = c.Lz / c.nz;
  h.inv_dx = 1.0 / h.dx; h.inv_dy = 1.0 / h.dy; h.inv_dz = 1.0 / h.dz;
  h.dt = c.dt;
  h.inv_dt = 1.0 / c.dt;
  // SpectralGrid scales (physics/spectral_state.py:112-133)
  h.dct_scale = (h.dx * h.dy) * std::sqrt((double)(c.nx * c.ny) / (c.Lx * c.Ly));
  h.recon_scale = std::sqrt((double)(c.nx * c.ny)) / std::sqrt(c.Lx * c.Ly);
  h.sqrt_dV = std::sqrt(h.dx * h.dy * h.dz);
  h.n_elements = (double)h.V;
  h.kbar = c.k;
  h.abar = c.rho * c.cp;
  h.T0 = c.T0;
  h.h_top = c.h_top;
  h.h_bottom = c.h_bottom;
  // evaporation constants (physics/spectral_cpu_kernels.py:150-151)
  h.evap_f1 = 0.82 * c.dH_LV * c.Pa / std::sqrt(2 * M_PI * c.R_v);
  h.evap_f2 = c.dH_LV / (c.R_v * c.T_boil);
  h.T_boil = c.T_boil;
  h.T_liquidus = c.T_liquidus;
  h.T_solidus = c.T_solidus;
  h.degenerate_band = !(c.T_liquidus > c.T_solidus);
  h.band_inv = h.degenerate_band ? 0.0 : 1.0 / (c.T_liquidus - c.T_solidus);
  h.latent_factor = -c.rho * c.L_f / c.dt;
  h.L_f = c.L_f;
  h.r_x = c.r_x; h.r_y = c.r_y;
  h.absorptivity = c.absorptivity;
  h.order = c.order;
  h.area_factor = c.area_factor;
  h.omega = c.omega;
  h.tol = c.tol;
  if (box) {
    // FineMeshState.__init__ (physics/spectral_state.py:189-227), in its operation order
    const double r = (double)c.box_refinement;
    h.dxf = h.dx / r; h.dyf = h.dy / r; h.dzf = h.dz / r;
    const double fx = std::ceil(c.Lx / h.dxf), fy = std::ceil(c.Ly / h.dyf), fz = std::ceil(c.box_size[2] / h.dzf);
    const double bx = std::ceil(c.box_size[0] / h.dxf), by = std::ceil(c.box_size[1] / h.dyf);
    if (!(fx <= 65536 && fy <= 65536 && fz <= 65536))
      return fail(SGH_ERR_INVALID, "fine box grid exceeds 65536 cells on an axis");
    h.fx = (int)fx; h.fy = (int)fy; h.fz = (int)fz;
    h.xb = std::min((int)bx, h.fx);
    h.yb = std::min((int)by, h.fy);
    h.zb = std::min((int)fz, h.fz);
    h.dV_fine = h.dxf * h.dyf * h.dzf;
    if (h.xb < 1 || h.yb < 1 || h.zb < 1) return fail(SGH_ERR_INVALID, "fine box is empty");
    const long long nb = (long long)h.zb * h.yb * h.xb;
    const long long lim = 1LL << 30;
    if (nb > lim || (long long)(h.zb + 1) * h.S > lim || (long long)h.zb * h.ny * h.xb > lim ||
        (long long)h.fx * h.nx > lim || (long long)h.fy * h.ny > lim)
      return fail(SGH_ERR_INVALID, "fine box too large (a box array exceeds 2^30 elements)");
    h.Nb = (int)nb;
  }
  if (c.has_model) {
    h.prog[P_K_SOLID] = c.k_solid;
    h.prog[P_K_LIQUID] = c.k_liquid;
    h.prog[P_RHO_SOLID] = c.rho_solid;
    h.prog[P_RHO_LIQUID] = c.rho_liquid;
    h.prog[P_C_SOLID] = c.c_solid;
    h.prog[P_C_LIQUID] = c.c_liquid;
    for (int i = 0; i < P_COUNT; ++i)
      h.affine[i] = program_affine(h.prog[i], &h.aff_a[i], &h.aff_b[i]) ? 1 : 0;
  }

  p->nparts_relax = std::min(RELAX_BLOCKS_MAX, cdiv(h.V, EW_THREADS));
  p->nparts_las = cdiv(h.S, EW_THREADS);
  p->nparts_surf = axis_blocks(h.ny, 1, h.nx);
  const int nparts_axis = axis_blocks(h.nz, 1, h.S);

  Layout L;
  const size_t V8 = sizeof(double) * (size_t)h.V, S8 = sizeof(double) * (size_t)h.S;
  p->o_params = L.take(sizeof(DevParams));
  p->o_ctrl = L.take(sizeof(Ctrl));
  p->o_mx = L.take(sizeof(double) * c.nx * c.nx);
  p->o_mxt = L.take(sizeof(double) * c.nx * c.nx);
  p->o_my = L.take(sizeof(double) * c.ny * c.ny);
  p->o_myt = L.take(sizeof(double) * c.ny * c.ny);
  p->o_mz = L.take(sizeof(double) * c.nz * c.nz);
  p->o_mzt = L.take(sizeof(double) * (c.nz + 2) * c.nz);  // + top and bottom surface rows
  p->o_xc = L.take(sizeof(double) * c.nx);
  p->o_yc = L.take(sizeof(double) * c.ny);
  p->o_ct = L.take(sizeof(double) * c.nz);
  p->o_cb = L.take(sizeof(double) * c.nz);
  p->o_K = L.take(V8);
  p->o_KK = L.take(V8);
  p->o_a = L.take(V8);
  p->o_aK = L.take(V8);
  p->o_trial = L.take(V8);
  p->o_Tprev = L.take(V8);
  p->o_Qm = L.take(V8);
  const size_t VX8 = sizeof(double) * (size_t)h.S * (c.nz + 2);  // volume + face slabs
  p->o_t1 = L.take(VX8);
  p->o_t2 = L.take(VX8);
  p->o_vol = L.take(VX8);
  p->o_kp = L.take(V8);
  p->o_qlas = L.take(S8);
  p->o_qnet = L.take(S8);
  p->o_qev = L.take(S8);
  p->o_qevold = L.take(S8);
  p->o_Stop = L.take(S8);
  p->o_Sbot = L.take(S8);
  p->o_f1 = L.take(S8);
  p->o_f2 = L.take(S8);
  p->o_Tsurf = L.take(S8);
  p->o_A = L.take(S8);
  p->o_prelax = L.take(sizeof(double) * 2 * std::max(p->nparts_relax, nparts_axis));
  p->o_plas = L.take(sizeof(double) * p->nparts_las);
  p->o_psurf = L.take(sizeof(double) * 2 * std::max(p->nparts_surf, axis_blocks(h.nz + 1, 1, h.S)));
  p->hist_cap = std::max(1, std::min(c.max_iter, SGH_PICARD_HISTORY_MAX));
  p->o_hist = L.take(sizeof(double) * 2 * p->hist_cap);
  p->face_space = !latent && !prop_corr && !box;
  if (box) {
    p->box_z0 = c.Lz - c.box_size[2];
    const size_t B8 = sizeof(double) * (size_t)h.Nb;
    p->o_bx = L.take(sizeof(double) * (size_t)h.fx * h.nx);
    p->o_by = L.take(sizeof(double) * (size_t)h.fy * h.ny);
    p->o_bzi = L.take(sizeof(double) * (size_t)(h.zb + 1) * h.nz);
    p->o_bzf = L.take(sizeof(double) * (size_t)h.nz * h.zb);
    p->o_wxi = L.take(sizeof(double) * (size_t)h.xb * h.nx);
    p->o_wxf = L.take(sizeof(double) * (size_t)h.xb * h.nx);
    p->o_wyi = L.take(sizeof(double) * (size_t)h.yb * h.ny);
    p->o_wyf = L.take(sizeof(double) * (size_t)h.yb * h.ny);
    p->o_bt1 = L.take(sizeof(double) * (size_t)(h.zb + 1) * h.S);
    p->o_bt2 = L.take(sizeof(double) * (size_t)h.zb * h.ny * h.xb);
    p->o_Qbox = L.take(B8);
    p->o_Tpb = L.take(B8);
    p->o_Qpb = L.take(B8);
    p->o_Tsh = L.take(B8);
    p->o_Qsh = L.take(B8);
  }
  p->nparts_n1 = cdiv(h.S, EW_THREADS);
  p->nparts_fs = std::min(RELAX_BLOCKS_MAX, cdiv(h.S, EW_THREADS));
  p->o_fsF = L.take(S8 * 4);
  p->o_fsW = L.take(S8 * 6);
  p->o_sigma = L.take(S8);
  p->o_beta = L.take(S8);
  p->o_Ab = L.take(S8);
  p->o_pn1 = L.take(sizeof(double) * p->nparts_n1);
  if (c.precision == SGH_PRECISION_MIXED) {
    // each matrix with the largest (rows, contraction length) its passes use
    auto plane = [&](size_t mat, int rows, int k, bool per_step = false) {
      p->plane_specs.push_back({mat, rows, k, L.take(umma::pair_bytes<AXU_M>(rows, k)), per_step});
    };
    plane(p->o_mx, h.nx, h.nx);
    plane(p->o_mxt, h.nx, h.nx);
    plane(p->o_my, h.ny, h.ny);
    plane(p->o_myt, h.ny, h.ny);
    plane(p->o_mz, h.nz, h.nz);
    plane(p->o_mzt, h.nz + 2, h.nz);
    if (box) {
      plane(p->o_bzi, h.zb + 1, h.nz);
      plane(p->o_wxi, h.xb, h.nx, true);
      plane(p->o_wyi, h.yb, h.ny, true);
      plane(p->o_wyf, h.ny, h.yb, true);
      plane(p->o_wxf, h.nx, h.xb, true);
      plane(p->o_bzf, h.nz, h.zb);
    }
  }
  p->ws_need = L.off;
  *out = p;
  return SGH_OK;
}

int sgh_plan_destroy(sgh_plan* p) {
  if (!p) return SGH_OK;
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  if (p->cs1) cudaStreamDestroy(p->cs1);
  if (p->cs2) cudaStreamDestroy(p->cs2);
  delete p;
  return SGH_OK;
}

int sgh_plan_workspace_bytes(const sgh_plan* p, uint64_t* bytes) {
  if (!p || !bytes) return fail(SGH_ERR_INVALID, "null argument");
  *bytes = p->ws_need;
  return SGH_OK;
}

int sgh_plan_bind(sgh_plan* p, void* workspace, uint64_t bytes, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !workspace) return fail(SGH_ERR_INVALID, "null argument");
  if (p->bound) return fail(SGH_ERR_STATE, "plan is already bound");
  if (bytes < p->ws_need) return fail(SGH_ERR_WORKSPACE, "workspace is smaller than sgh_plan_workspace_bytes()");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(SGH_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  p->ws = static_cast<char*>(workspace);
  g_umma_err = umma_err_of(p);  // the policy above was made before the workspace existed
  const DevParams& h = p->hp;
  SGH_CK(cudaMemcpyAsync(p->P(), &h, sizeof(DevParams), cudaMemcpyHostToDevice, s));
  SGH_CK(cudaMemsetAsync(p->ctrl(), 0, sizeof(Ctrl), s));
  k_ctrl_history<<<1, 1, 0, s>>>(p->ctrl(), p->d(p->o_hist), p->hist_cap);
  struct { int n; size_t m, mt; } mats[3] = {{h.nx, p->o_mx, p->o_mxt}, {h.ny, p->o_my, p->o_myt},
                                             {h.nz, p->o_mz, p->o_mzt}};
  for (auto& m : mats)
    k_dct_matrix<<<cdiv((long)m.n * m.n, EW_THREADS), EW_THREADS, 0, s>>>(m.n, p->d(m.m), p->d(m.mt));
  const int gmax = cdiv(std::max(std::max(h.nx, h.ny), h.nz), EW_THREADS);
  k_grid_tables<<<gmax, EW_THREADS, 0, s>>>(p->P(), p->d(p->o_xc), p->d(p->o_yc), p->d(p->o_ct), p->d(p->o_cb),
                                            p->d(p->o_mzt));
  const sgh_config& c = p->cfg;
  const double alpha = c.k / (c.rho * c.cp);
  k_propagators<<<cdiv(h.V, EW_THREADS), EW_THREADS, 0, s>>>(p->P(), alpha, c.rho * c.cp, p->d(p->o_K),
                                                             p->d(p->o_KK));
  SGH_CK(cudaMemsetAsync(p->ws + p->o_Sbot, 0, sizeof(double) * h.S, s));
  if (h.box) {
    k_fine_basis<<<cdiv((long)h.fx * h.nx, EW_THREADS), EW_THREADS, 0, s>>>(h.nx, h.fx, c.Lx, h.dxf, 0.0,
                                                                          p->d(p->o_bx), nullptr);
    k_fine_basis<<<cdiv((long)h.fy * h.ny, EW_THREADS), EW_THREADS, 0, s>>>(h.ny, h.fy, c.Ly, h.dyf, 0.0,
                                                                          p->d(p->o_by), nullptr);
    k_fine_basis<<<cdiv((long)h.zb * h.nz, EW_THREADS), EW_THREADS, 0, s>>>(h.nz, h.zb, c.Lz, h.dzf, p->box_z0,
                                                                          p->d(p->o_bzi), p->d(p->o_bzf));
    // face row of the z reconstruction matrix: the top-surface weights
    SGH_CK(cudaMemcpyAsync(p->d(p->o_bzi) + (size_t)h.zb * h.nz, p->d(p->o_ct), sizeof(double) * h.nz,
                           cudaMemcpyDeviceToDevice, s));
  }
  if (p->face_space)
    k_fs_weights<<<cdiv(h.S, EW_THREADS), EW_THREADS, 0, s>>>(p->P(), p->d(p->o_KK), p->d(p->o_ct),
                                                              p->d(p->o_cb), p->d(p->o_fsW));
  // BF16 pair planes of the matrices (mixed plans), once the matrices exist
  // (the window bases' planes are rebuilt with the window every step)
  p->planes.clear();
  for (const auto& q : p->plane_specs) {
    if (!q.per_step) build_plane(p, q, s);
    p->planes.push_back({p->d(q.mat), p->ws + q.off, q.rows, q.k});
  }
  p->bound_planes = true;
  g_umma_planes = planes_of(p);
  g_umma_nplanes = nplanes_of(p);
  SGH_CK(cudaGetLastError());
  SGH_CK(cudaStreamSynchronize(s));
  SGH_CK(cudaStreamCreateWithFlags(&p->cs1, cudaStreamNonBlocking));
  SGH_CK(cudaStreamCreateWithFlags(&p->cs2, cudaStreamNonBlocking));
  const int rc = capture(p);
  if (rc) return rc;
  p->bound = true;
  const int rr = sgh_state_reset(p, stream);
  if (rr) return rr;
  SGH_CK(cudaStreamSynchronize(s));
  return SGH_OK;
}

int sgh_plan_launch_counts(const sgh_plan* p, int32_t* pre, int32_t* per_iter, int32_t* post) {
  if (!p || !pre || !per_iter || !post) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  *pre = p->n_pre + 1;  // + the launch-setup kernel of sgh_step / sgh_run
  *per_iter = p->n_iter;
  *post = p->n_post;
  return SGH_OK;
}

int sgh_plan_buffer(const sgh_plan* p, int32_t which, void** ptr, uint64_t* bytes) {
  if (!p || !ptr) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->ws) return fail(SGH_ERR_STATE, "plan is not bound");
  const size_t V8 = sizeof(double) * (size_t)p->hp.V, S8 = sizeof(double) * (size_t)p->hp.S;
  size_t off, n;
  switch (which) {
    case SGH_BUF_MODES: off = p->o_a; n = V8; break;
    case SGH_BUF_K: off = p->o_K; n = V8; break;
    case SGH_BUF_KK: off = p->o_KK; n = V8; break;
    case SGH_BUF_T_PREV: off = p->o_Tprev; n = V8; break;
    case SGH_BUF_Q_EVAP_OLD: off = p->o_qevold; n = S8; break;
    case SGH_BUF_Q_MODES: off = p->o_Qm; n = V8; break;
    case SGH_BUF_SURFACE: off = p->o_Tsurf; n = S8; break;
    case SGH_BUF_SCRATCH: off = p->o_vol; n = V8; break;
    case SGH_BUF_BOX_T_PREV:
    case SGH_BUF_BOX_Q_PREV:
    case SGH_BUF_BOX_BX:
    case SGH_BUF_BOX_BY:
    case SGH_BUF_BOX_BZ: {
      const DevParams& h = p->hp;
      if (!h.box) return fail(SGH_ERR_STATE, "box buffers exist in box mode only");
      if (which == SGH_BUF_BOX_T_PREV) { off = p->o_Tpb; n = sizeof(double) * (size_t)h.Nb; }
      else if (which == SGH_BUF_BOX_Q_PREV) { off = p->o_Qpb; n = sizeof(double) * (size_t)h.Nb; }
      else if (which == SGH_BUF_BOX_BX) { off = p->o_bx; n = sizeof(double) * (size_t)h.fx * h.nx; }
      else if (which == SGH_BUF_BOX_BY) { off = p->o_by; n = sizeof(double) * (size_t)h.fy * h.ny; }
      else { off = p->o_bzi; n = sizeof(double) * (size_t)(h.zb + 1) * h.nz; }
      break;
    }
    default: return fail(SGH_ERR_INVALID, "unknown buffer id");
  }
  *ptr = p->ws + off;
  if (bytes) *bytes = n;
  return SGH_OK;
}

int sgh_state_reset(sgh_plan* p, void* stream) {
  if (!p || !p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = std::max(p->hp.V, p->hp.S);
  k_reset<<<cdiv(n, EW_THREADS), EW_THREADS, 0, s>>>(p->P(), p->ctrl(), p->d(p->o_a), p->d(p->o_Tprev),
                                                     p->d(p->o_qevold), p->d(p->o_qev), p->d(p->o_Qm));
  SGH_CK(cudaGetLastError());
  if (p->hp.box) {
    // no window yet: zero window bases (physics/spectral_state.py:221-225), no history
    const DevParams& h = p->hp;
    const size_t wx = sizeof(double) * (size_t)h.xb * h.nx, wy = sizeof(double) * (size_t)h.yb * h.ny;
    const size_t B8 = sizeof(double) * (size_t)h.Nb;
    SGH_CK(cudaMemsetAsync(p->ws + p->o_wxi, 0, wx, s));
    SGH_CK(cudaMemsetAsync(p->ws + p->o_wxf, 0, wx, s));
    SGH_CK(cudaMemsetAsync(p->ws + p->o_wyi, 0, wy, s));
    SGH_CK(cudaMemsetAsync(p->ws + p->o_wyf, 0, wy, s));
    SGH_CK(cudaMemsetAsync(p->ws + p->o_Tpb, 0, B8, s));
    SGH_CK(cudaMemsetAsync(p->ws + p->o_Qpb, 0, B8, s));
    SGH_CK(cudaMemsetAsync(p->ws + p->o_Qbox, 0, B8, s));
  }
  return SGH_OK;
}

int sgh_step(sgh_plan* p, const sgh_laser* laser, sgh_step_out* out, void* stream) {
  if (!p || !laser) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_run_setup<<<1, 1, 0, s>>>(p->ctrl(), *laser, nullptr, nullptr, 1);
  SGH_CK(cudaGetLastError());
  SGH_CK(cudaGraphLaunch(p->exec, s));
  if (out) SGH_CK(cudaMemcpyAsync(out, &p->ctrl()->out, sizeof(sgh_step_out), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaStreamSynchronize(s));
  return SGH_OK;
}

int sgh_step_eager(sgh_plan* p, const sgh_laser* laser, sgh_step_out* out, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !laser) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_run_setup<<<1, 1, 0, s>>>(p->ctrl(), *laser, nullptr, nullptr, 1);
  enqueue_pre(p, s);
  for (int it = 0; it < p->hp.max_iter; ++it) {
    enqueue_picard(p, s, 0, 0);
    int stop = 0;
    SGH_CK(cudaMemcpyAsync(&stop, &p->ctrl()->stop, sizeof(int), cudaMemcpyDeviceToHost, s));
    SGH_CK(cudaStreamSynchronize(s));
    if (stop) break;
  }
  enqueue_post(p, s, 0, 0);
  SGH_CK(cudaGetLastError());
  if (out) SGH_CK(cudaMemcpyAsync(out, &p->ctrl()->out, sizeof(sgh_step_out), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaStreamSynchronize(s));
  return SGH_OK;
}

int sgh_run(sgh_plan* p, const sgh_laser* lasers_dev, int32_t n_steps, sgh_step_out* outs_dev, void* stream) {
  if (!p || !lasers_dev) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  if (n_steps < 0) return fail(SGH_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return SGH_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  sgh_laser dummy = {};
  k_run_setup<<<1, 1, 0, s>>>(p->ctrl(), dummy, lasers_dev, outs_dev, n_steps);
  SGH_CK(cudaGetLastError());
  SGH_CK(cudaGraphLaunch(p->exec, s));
  return SGH_OK;
}

int sgh_dct3d(sgh_plan* p, int32_t kind, const double* in, double* out, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !in || !out) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  if (kind != 2 && kind != 3) return fail(SGH_ERR_INVALID, "kind must be 2 (DCT_II) or 3 (IDCT_II)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  volume_pass3(p, in, kind == 3, EpiStore{out, 1.0, nullptr}, p->d(p->o_t1), p->d(p->o_t2), s);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_surface_temperature(sgh_plan* p, const double* modes, int32_t top, double* out, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !modes || !out) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  face_idct2(p, modes, p->d(top ? p->o_ct : p->o_cb), EpiFaceTemperature{point_phys(p->hp, p->P()), out, nullptr}, s);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_project_volume(sgh_plan* p, const double* field, double* modes, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !field || !modes) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  volume_pass3(p, field, false, EpiStore{modes, p->hp.sqrt_dV, nullptr}, p->d(p->o_t1), p->d(p->o_t2), s);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_reconstruct_volume(sgh_plan* p, const double* modes, double* field, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !field || !modes) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  volume_pass3(p, modes, true, EpiDiv{field, p->hp.sqrt_dV, nullptr}, p->d(p->o_t1), p->d(p->o_t2), s);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_state_flags(sgh_plan* p, int32_t* flags, void* stream) {
  if (!p || !flags) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t v[2];
  SGH_CK(cudaMemcpyAsync(&v[0], &p->ctrl()->have_qprev, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaMemcpyAsync(&v[1], &p->ctrl()->have_tprev, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaStreamSynchronize(s));
  *flags = (v[0] ? SGH_STATE_HAVE_Q_MODES : 0) | (v[1] ? SGH_STATE_HAVE_BOX : 0);
  return SGH_OK;
}

int sgh_state_set_flags(sgh_plan* p, int32_t flags, void* stream) {
  if (!p) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  if (flags & ~(SGH_STATE_HAVE_Q_MODES | SGH_STATE_HAVE_BOX)) return fail(SGH_ERR_INVALID, "unknown flag bits");
  if ((flags & SGH_STATE_HAVE_BOX) && !p->hp.box) return fail(SGH_ERR_INVALID, "box history flag on a grid-mode plan");
  k_set_flags<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(p->ctrl(), flags);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_box_geometry(const sgh_plan* p, sgh_box_geom* out) {
  if (!p || !out) return fail(SGH_ERR_INVALID, "null argument");
  const DevParams& h = p->hp;
  if (!h.box) return fail(SGH_ERR_STATE, "plan is not in box mode");
  out->n_box[0] = h.xb; out->n_box[1] = h.yb; out->n_box[2] = h.zb;
  out->n_fine_total[0] = h.fx; out->n_fine_total[1] = h.fy; out->n_fine_total[2] = h.fz;
  out->d_fine[0] = h.dxf; out->d_fine[1] = h.dyf; out->d_fine[2] = h.dzf;
  out->dV_fine = h.dV_fine;
  out->z0 = p->box_z0;
  return SGH_OK;
}

int sgh_picard_history(sgh_plan* p, double* out, int32_t cap, int32_t* n_iter, void* stream) {
  if (!p || !out || !n_iter || cap < 0) return fail(SGH_ERR_INVALID, "null argument or negative cap");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t it = 0;
  SGH_CK(cudaMemcpyAsync(&it, &p->ctrl()->iter, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaStreamSynchronize(s));
  const int n = std::min(std::min(it, p->hist_cap), (int)cap);
  if (n > 0) {
    SGH_CK(cudaMemcpyAsync(out, p->ws + p->o_hist, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s));
    SGH_CK(cudaStreamSynchronize(s));
  }
  *n_iter = it;
  return SGH_OK;
}

int sgh_box_window(sgh_plan* p, int32_t* i0, void* stream) {
  if (!p || !i0) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  if (!p->hp.box) return fail(SGH_ERR_STATE, "plan is not in box mode");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int32_t w[2];
  SGH_CK(cudaMemcpyAsync(&w[0], &p->ctrl()->box_i0x, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaMemcpyAsync(&w[1], &p->ctrl()->box_i0y, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  SGH_CK(cudaStreamSynchronize(s));
  i0[0] = w[0];
  i0[1] = w[1];
  return SGH_OK;
}

int sgh_box_temperature(sgh_plan* p, const double* modes, double* out, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !modes || !out) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  if (!p->hp.box) return fail(SGH_ERR_STATE, "plan is not in box mode");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  box_zpass(p, modes, false, s);
  box_xy(p, EpiStore{out, 1.0, nullptr}, s);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_box_project(sgh_plan* p, const double* field_box, double* modes, void* stream) {
  AxisPolicy policy(p ? p->cfg.axis_min_ctas : 0, p ? p->cfg.axis_cuda_cores : 0, plan_mixed(p), umma_err_of(p),
                    plan_fp32(p), planes_of(p), nplanes_of(p));
  if (!p || !field_box || !modes) return fail(SGH_ERR_INVALID, "null argument");
  if (!p->bound) return fail(SGH_ERR_STATE, "plan is not bound");
  if (!p->hp.box) return fail(SGH_ERR_STATE, "plan is not in box mode");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  box_project(p, field_box, EpiStore{modes, p->hp.dV_fine, nullptr}, s);
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

namespace {
struct DctnLayout {
  int n[3] = {1, 1, 1};   // (n0, n1, n2), n2 fastest; unused leading axes are 1
  int ndim = 0;
  size_t o_mat[3] = {0, 0, 0}, o_t1 = 0, o_t2 = 0, total = 0;
};

int dctn_layout(int32_t ndim, const int32_t* shape, DctnLayout* L) {
  if (ndim < 1 || ndim > 3 || !shape) return fail(SGH_ERR_INVALID, "ndim must be 1, 2 or 3");
  long long vol = 1;
  for (int i = 0; i < ndim; ++i) {
    if (shape[i] < 1 || shape[i] > 4096) return fail(SGH_ERR_INVALID, "axis length must be in [1, 4096]");
    vol *= shape[i];
  }
  if (vol > (1LL << 28)) return fail(SGH_ERR_INVALID, "array exceeds 2^28 elements");
  L->ndim = ndim;
  for (int i = 0; i < ndim; ++i) L->n[3 - ndim + i] = shape[i];
  Layout lay;
  for (int a = 0; a < 3; ++a) L->o_mat[a] = lay.take(sizeof(double) * 2 * L->n[a] * L->n[a]);
  L->o_t1 = lay.take(sizeof(double) * vol);
  L->o_t2 = lay.take(sizeof(double) * vol);
  L->total = lay.off;
  return SGH_OK;
}
}  // namespace

int sgh_dctn_workspace_bytes(int32_t ndim, const int32_t* shape, uint64_t* bytes) {
  if (!bytes) return fail(SGH_ERR_INVALID, "null argument");
  DctnLayout L;
  const int rc = dctn_layout(ndim, shape, &L);
  if (rc) return rc;
  *bytes = L.total;
  return SGH_OK;
}

int sgh_dctn(int32_t kind, int32_t ndim, const int32_t* shape, const double* in, double* out,
             void* workspace, uint64_t bytes, void* stream) {
  if (!in || !out || !workspace) return fail(SGH_ERR_INVALID, "null argument");
  if (kind != 2 && kind != 3) return fail(SGH_ERR_INVALID, "kind must be 2 (DCT_II) or 3 (IDCT_II)");
  DctnLayout L;
  const int rc = dctn_layout(ndim, shape, &L);
  if (rc) return rc;
  if (bytes < L.total) return fail(SGH_ERR_WORKSPACE, "workspace is smaller than sgh_dctn_workspace_bytes()");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(SGH_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  const double* mats[3];
  for (int a = 0; a < 3; ++a) {
    const int N = L.n[a];
    double* M = reinterpret_cast<double*>(ws + L.o_mat[a]);
    k_dct_matrix<<<cdiv((long)N * N, EW_THREADS), EW_THREADS, 0, s>>>(N, M, M + (size_t)N * N);
    mats[a] = (kind == 2) ? M : M + (size_t)N * N;
  }
  double* t1 = reinterpret_cast<double*>(ws + L.o_t1);
  double* t2 = reinterpret_cast<double*>(ws + L.o_t2);
  const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
  // passes over the last ndim axes, fastest first; the final pass writes out
  const int first = 3 - L.ndim;
  const double* src = in;
  double* bufs[2] = {t1, t2};
  int nb = 0;
  if (L.ndim == 1 && in == out) {  // a single pass must not read what it writes
    SGH_CK(cudaMemcpyAsync(t2, in, sizeof(double) * (size_t)n2, cudaMemcpyDeviceToDevice, s));
    src = t2;
  }
  for (int a = 2; a >= first; --a) {
    double* dst = (a == first) ? out : bufs[nb++ & 1];
    const int N = L.n[a];
    const int A = (a == 2) ? n0 * n1 : (a == 1 ? n0 : 1);
    const int B = (a == 2) ? 1 : (a == 1 ? n2 : n1 * n2);
    launch_axis(src, mats[a], N, N, A, B, EpiStore{dst, 1.0, nullptr}, s);
    src = dst;
  }
  SGH_CK(cudaGetLastError());
  return SGH_OK;
}

// ---------------------------------------------------------------------------
// allocation-free DCT
// ---------------------------------------------------------------------------
// Scratch of sgh_dctn_noalloc: a fixed array in the module's global memory.
// Every device that loads the library holds it (SGH_NOALLOC_SCRATCH_BYTES)
// until the process exits. The host reaches it only through the address that
// cudaGetSymbolAddress returns for the current device; the symbol name itself
// is not a device address in host code.
static __device__ __align__(256) double g_noalloc_scratch[SGH_NOALLOC_SCRATCH_BYTES / sizeof(double)];

int sgh_dctn_noalloc(int32_t kind, int32_t ndim, const int32_t* shape, const double* in, double* out,
                     void* stream) {
  if (!in || !out) return fail(SGH_ERR_INVALID, "null argument");
  if (kind != 2 && kind != 3) return fail(SGH_ERR_INVALID, "kind must be 2 (DCT_II) or 3 (IDCT_II)");
  DctnLayout L;
  const int rc = dctn_layout(ndim, shape, &L);
  if (rc) return rc;
  if (L.total > SGH_NOALLOC_SCRATCH_BYTES)
    return fail(SGH_ERR_WORKSPACE,
                "array too large for sgh_dctn_noalloc: needs " + std::to_string(L.total) +
                    " bytes of scratch, the built-in scratch holds " +
                    std::to_string((unsigned long long)SGH_NOALLOC_SCRATCH_BYTES) + "; use sgh_dctn");
  // The device address of the scratch on the current device, looked up on
  // every call (no allocation, and nothing cached that a context reset could
  // leave stale).
  void* scratch = nullptr;
  SGH_CK(cudaGetSymbolAddress(&scratch, g_noalloc_scratch));
  if (!scratch) return fail(SGH_ERR_CUDA, "cudaGetSymbolAddress returned a null scratch address");
  return sgh_dctn(kind, ndim, shape, in, out, scratch, SGH_NOALLOC_SCRATCH_BYTES, stream);
}

}  // extern "C"
