// sgh_batch.cu -- many instances of uneven size stepped together.
//
// Every stage of the time step runs as ONE launch over all slots of a batch.
// Work is decomposed per slot: element/column kernels give each slot
// ceil(S_i / 256) blocks, face transforms give each slot its tiles (FP64) or
// 128-row x 128-column tiles (mixed); a block reads its slot from a block ->
// slot table. Per-slot reductions (P_laser, Picard norms, surface max) are
// per-block partials summed slot by slot in a fixed order.
//
// The physics is the face-space Picard form (see sgh_b200.cu): every iterate
// of a slot is aK + KK Ct[p] sigma[y,x], so each step reads the modes twice
// (K a and the face sums; the commit) and the Picard loop runs on faces: an
// inverse 2-D transform with the evaporation epilogue, a forward 2-D
// transform, and the relaxation, whose last blocks also run the convergence
// test. The loop is a conditional graph node that repeats while any slot is
// still iterating; converged (or inactive) slots skip every kernel of the
// body, so a slot's result does not depend on what else is in the batch.
//
// Volume state is FP64 modes with stored K and KK (plain), or FP32 modes only
// (mixed: K and KK formed in registers from per-axis FP64 tables, the mode
// update in FP32). Face fields and norms are FP64 in both; the face sums and
// weights (Zt, Yt, W_tt, Q_tt) are FP32 in mixed batches, where the face
// transforms run on the tensor cores from split-BF16 operand planes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "sgh_b200.h"
#include "sgh_axis.cuh"
#include "sgh_device.cuh"
#include "sgh_umma.cuh"

namespace sgh {
namespace batch {

constexpr int BT = 256;   // threads of element / column / face kernels
constexpr int CT = 1024;  // threads of the per-slot control kernels
constexpr int RPT = 8;    // elements per thread of the relaxation
constexpr int RB = RPT * BT;
constexpr int VOL_FLUSH = 8;  // z-planes per FP32 partial sum of the mixed volume passes
constexpr int RING_TABMAX = 256;  // largest nz of the ring-staged volume pass (its per-plane table)

struct BSlot {
  int nx, ny, nz, S;
  long long V;
  int max_iter, cell_integrated;
  long long vol;   // element offset of this slot in the volume arenas
  long long face;  // element offset in the face arenas
  int zoff;        // offset in the Ct table
  int eoff;        // offset of the slot's 1-D tables, each over x (nx), y (ny), z (nz):
                   // decay E = exp(-alpha dt k^2), D = 1 - E, L = kbar k^2
  int mx, my;      // element offsets of the x / y DCT matrices (M, then M^T)
  int blk0, nblk;  // element / column blocks
  int rblk0, nrblk;  // relaxation blocks (RB elements)
  int tile0, ntile;  // face transform tiles
  int vblk0, nvblk;  // volume blocks (setup kernels)
  int utile0, nutile;  // tensor-core face tiles (mixed precision)
  long long xa;        // byte offset of the slot's face planes (rows y, k = x) in the xa / xq arenas
  long long mpx, mpy;  // byte offsets of the forward x / y matrix planes (inverse at + mp_inv)
  long long mpx_inv, mpy_inv;
  long long x1;        // byte offset of the slot's x1 plane (x-pass result, y-pass B operand)
  double dx, dy, dt, Lx, Ly, Lz;
  double dct_scale, recon_scale, n_elements;
  double T0, evap_f1, evap_f2, T_boil, T_liquidus;
  double r_x, r_y, absorptivity, order, area_factor;
  double omega, tol;
  double k, rho, cp;
};

struct BState {
  sgh_laser laser;
  const sgh_laser* table;
  sgh_step_out* outs;
  int n_steps, step, active, iters;
  int iter, done, status;
  unsigned tickets;  // kb_relax blocks of this slot done in the current launch
  int pass1_ready;   // the commit already formed the next step's face sums
  int pad2;
  double I0, shift_x, shift_y, rel_err;
  sgh_step_out last;
};

struct BGlobal {
  int steps_left;
  int umma_err;     // nonzero once a tensor-core wait expired
  int picard_any;   // some slot is still iterating (read by the eager step)
  unsigned slots_done;   // slots finished in the current kb_relax launch (back to 0 after it)
  int n_iter_slots;      // slots iterating in the current Picard iteration
  unsigned wait_limit;   // polls of the tensor-core data waits (0: umma::WAIT_LIMIT)
  int stall_test;        // 1: every face y-pass CTA first waits on a barrier nothing completes
  int pad;
};

// Device view of a bound batch (passed by value to every kernel).
struct BView {
  const BSlot* slot;
  BState* st;
  BGlobal* g;
  const int* blk_slot;    // slot of each element / column block
  const int* rblk_slot;   // slot of each relaxation block
  const int* tile_slot;   // slot of each FP64 face-transform tile
  const int* vblk_slot;   // slot of each volume block
  const int* utile_slot;  // slot of each tensor-core face tile
  char* xa;               // operand pair planes (mixed precision; null otherwise):
  char* xq;               //   xa = A = Zt + W_tt sigma (inverse transform input), xq = q_net (forward)
  char* x1;               //   x1 = the x-pass result of the face transform in flight
  const char* mp;         // DCT matrix pair planes
  const double* mats;
  const double* Ct;
  const double* E;        // 1-D decay tables exp(-alpha dt k_i^2) per slot and axis
  int n;
};

// Eight lanes 8g..8g+7 of a warp hold consecutive k = k0..k0+7 (k0 % 8 == 0)
// of one plane row; lane 8g writes the group's 16-byte hi and lo rows. Call
// from all 32 lanes; `store` is read on lane 8g only.
__device__ __forceinline__ void plane_put8_warp(char* plane, int r, int k0, int nkc, double val, bool store) {
  __nv_bfloat16 h, l;
  umma::split_bf16(val, h, l);
  const uint32_t hv = __bfloat16_as_ushort(h), lv = __bfloat16_as_ushort(l);
  const uint32_t hp = hv | (__shfl_down_sync(0xffffffffu, hv, 1) << 16);
  const uint32_t lp = lv | (__shfl_down_sync(0xffffffffu, lv, 1) << 16);
  const uint32_t h1 = __shfl_down_sync(0xffffffffu, hp, 2), l1 = __shfl_down_sync(0xffffffffu, lp, 2);
  const uint32_t h2 = __shfl_down_sync(0xffffffffu, hp, 4), l2 = __shfl_down_sync(0xffffffffu, lp, 4);
  const uint32_t h3 = __shfl_down_sync(0xffffffffu, hp, 6), l3 = __shfl_down_sync(0xffffffffu, lp, 6);
  if ((threadIdx.x & 7) == 0 && store) {
    const size_t o = umma::pair_off<umma::TM>(r, k0, nkc);
    *reinterpret_cast<uint4*>(plane + o) = make_uint4(hp, h1, h2, h3);
    *reinterpret_cast<uint4*>(plane + o + umma::pair_chunk_bytes<umma::TM>()) = make_uint4(lp, l1, l2, l3);
  }
}

// Face-plane element i = y * nx + x of slot sl (plane: the xa or xq pair
// arena, null in FP64 batches), written by a whole block of consecutive i (one
// slot per block). When nx % 8 == 0 every aligned group of 8 lanes is 8
// consecutive x of one row and goes out as one 16-byte store per part.
__device__ __forceinline__ void plane_put_yx(char* plane, const BSlot& sl, int y, int x, double val, bool valid) {
  if (!plane) return;
  const int nkc = (sl.nx + umma::KC - 1) / umma::KC;
  if ((sl.nx & 7) == 0)
    plane_put8_warp(plane + sl.xa, y, x, nkc, valid ? val : 0.0, valid);
  else if (valid)
    umma::pair_put<umma::TM>(plane + sl.xa, y, x, nkc, val);
}
__device__ __forceinline__ void plane_put_block(char* plane, const BSlot& sl, int i, double val, bool valid) {
  if (!plane) return;
  const int nkc = (sl.nx + umma::KC - 1) / umma::KC;
  const int y = i / sl.nx, x = i - (i / sl.nx) * sl.nx;
  if ((sl.nx & 7) == 0)
    plane_put8_warp(plane + sl.xa, y, x, nkc, valid ? val : 0.0, valid);
  else if (valid)
    umma::pair_put<umma::TM>(plane + sl.xa, y, x, nkc, val);
}

// ---------------------------------------------------------------------------
// setup
// ---------------------------------------------------------------------------

__global__ void kb_dct_matrix(int N, double* M) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * N) return;
  const int k = e / N, n = e - k * N;
  const long long m = ((long long)k * (2 * n + 1)) % (4LL * N);
  const double w = (k == 0) ? sqrt(1.0 / N) : sqrt(2.0 / N);
  const double v = w * cospi((double)m / (double)(2 * N));
  M[k * N + n] = v;
  M[(size_t)N * N + n * N + k] = v;
}

// BF16 hi/lo pair planes of an N x N DCT matrix (inv: its transpose), rows = the
// output index, k = the contracted index, in R-row chunks.
template <int R>
__global__ void kb_matrix_planes(int N, const double* M, int inv, char* plane) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * N) return;
  const int r = e / N, k = e - r * N;
  const double val = inv ? M[(size_t)k * N + r] : M[(size_t)r * N + k];
  umma::pair_put<R>(plane, r, k, (N + umma::KC - 1) / umma::KC, val);
}

// KK of one mode in the mixed-precision form, from per-axis tables (FP32):
// KK = (1 - Ex Ey Ez) / (kbar (qx^2 + qy^2 + qz^2)), and dt / (rho c) for the
// zero mode (precompute_K_KK, physics/spectral_state.py:405-413, with
// alpha rho c = kbar). The numerator is formed without cancellation as
// (1 - Ex Ey) + Ex Ey (1 - Ez), each 1 - E_axis an accurate -expm1 table
// entry, so the low modes (1 - K ~ 1e-4) keep full FP32 accuracy; the
// quotient is a fast FP32 division. Relative error a few 1e-7, the order of
// the FP32 rounding of a stored KK, at a handful of FP32 instructions per mode
// instead of 4 bytes of HBM traffic.
__device__ __forceinline__ double mode_kk(float dxy, float exy, float dz, float lxy, float lz,
                                          double dt_rc) {
  const float num = fmaf(exy, dz, dxy);
  const float den = lxy + lz;
  return den > 0.0f ? (double)__fdividef(num, den) : dt_rc;
}

// K, KK of every slot exactly as precompute_K_KK (physics/spectral_state.py:374-421),
// in FP64, stored as R (K and KK only when given); Ct tables; and per axis the
// 1-D tables E[i] = exp(-alpha dt k_i^2), D[i] = 1 - E[i] (as -expm1) and
// L[i] = kbar k_i^2. K = exp(-alpha dt (kx^2 + ky^2 + kz^2)) is exactly
// separable, K = Ex[x] Ey[y] Ez[z] (FP64), and KK follows from D, E and L
// (mode_kk): the mixed-precision form stores neither.
template <class R>
__global__ void __launch_bounds__(BT) kb_tables(BView v, R* K, R* KK, double* Ct, double* E) {
  const int b = blockIdx.x;
  const int s = v.vblk_slot[b];
  const BSlot& sl = v.slot[s];
  const long long i = (long long)(b - sl.vblk0) * BT + threadIdx.x;
  if (i < sl.V) {
    const int z = (int)(i / sl.S);
    const int r = (int)(i - (long long)z * sl.S);
    const int y = r / sl.nx, x = r - y * sl.nx;
    const double alpha = sl.k / (sl.rho * sl.cp);
    const double rho_cp = sl.rho * sl.cp;
    const double kz = M_PI * (double)z / sl.Lz;
    const double ky = M_PI * (double)y / sl.Ly;
    const double kx = M_PI * (double)x / sl.Lx;
    const double lam = alpha * (kz * kz + ky * ky + kx * kx);
    const double k = exp(-lam * sl.dt);
    if (K) K[sl.vol + i] = (R)k;
    const int nsum = sl.nx + sl.ny + sl.nz;
    const int axis_n[3] = {sl.nx, sl.ny, sl.nz};
    const double axis_L[3] = {sl.Lx, sl.Ly, sl.Lz};
    for (int ax = 0, base = 0; ax < 3; base += axis_n[ax], ++ax) {
      if (i < axis_n[ax]) {
        const double q = M_PI * (double)i / axis_L[ax];
        const double e = -(alpha * (q * q)) * sl.dt;
        E[sl.eoff + base + i] = exp(e);
        E[sl.eoff + nsum + base + i] = -expm1(e);
        E[sl.eoff + 2 * nsum + base + i] = sl.k * (q * q);
      }
    }
    if (KK) KK[sl.vol + i] = (R)((i == 0) ? sl.dt / rho_cp : ((k - 1.0) / (-lam)) / rho_cp);
    if (i < sl.nz) {
      const double c = (i == 0) ? sqrt(1.0 / sl.Lz) : sqrt(2.0 / sl.Lz);
      Ct[sl.zoff + i] = (i & 1) ? -c : c;
    }
  }
}

// Face weights from the stored KK: W_tt = sum Ct^2 KK, Q_tt = sum (KK Ct)^2.
template <class R>
__global__ void __launch_bounds__(BT) kb_weights(BView v, const R* KK, R* Wtt, R* Qtt) {
  const int b = blockIdx.x;
  const int s = v.blk_slot[b];
  const BSlot& sl = v.slot[s];
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  if (i >= sl.S) return;
  const int nsum = sl.nx + sl.ny + sl.nz;
  const double* E = v.E + sl.eoff;
  const double* D = E + nsum;
  const double* Lt = E + 2 * nsum;
  const int ix = i % sl.nx, iy = sl.nx + i / sl.nx, z0 = sl.nx + sl.ny;
  const float exy = (float)(E[ix] * E[iy]);
  const float dxy = (float)(D[ix] + E[ix] * D[iy]);
  const float lxy = (float)(Lt[ix] + Lt[iy]);
  const double dt_rc = sl.dt / (sl.rho * sl.cp);
  double w = 0.0, q = 0.0;
  for (int p = 0; p < sl.nz; ++p) {
    const double kk = KK ? (double)KK[sl.vol + (long long)p * sl.S + i]
                         : mode_kk(dxy, exy, (float)D[z0 + p], lxy, (float)Lt[z0 + p], dt_rc);
    const double ct = v.Ct[sl.zoff + p];
    w += ct * ct * kk;
    q += (kk * ct) * (kk * ct);
  }
  Wtt[sl.face + i] = (R)w;
  Qtt[sl.face + i] = (R)q;
}

// (Re)start one slot at the initial condition (solvers/spectral.py:176-180).
template <class R>
__global__ void __launch_bounds__(BT)
kb_slot_start(BView v, int s, R* a, double* q_evold, double* sigma, const sgh_laser* table,
              int n_steps, sgh_step_out* outs) {
  const BSlot& sl = v.slot[s];
  const long long i = (long long)blockIdx.x * BT + threadIdx.x;
  if (i < sl.V) a[sl.vol + i] = (R)((i == 0) ? sl.T0 * sqrt(sl.Lx * sl.Ly * sl.Lz) : 0.0);
  if (i < sl.S) {
    q_evold[sl.face + i] = 0.0;
    sigma[sl.face + i] = 0.0;
  }
  if (i == 0) {
    BState& st = v.st[s];
    st.table = table;
    st.outs = outs;
    st.n_steps = n_steps;
    st.step = 0;
    st.active = n_steps > 0 ? 1 : 0;
    st.iters = 0;
    st.done = 1;
    st.iter = 0;
    st.pass1_ready = 0;
  }
}

__global__ void kb_slot_stop(BView v, int s) { v.st[s].active = 0; }

// Resume one slot from state already written into its buffers (modes and
// q_evap_old, exported from another slot or batch): it continues at step
// `step` of its laser table. The next step forms its face sums from the
// stored modes (pass1_ready = 0), exactly as the commit would have.
__global__ void kb_slot_resume(BView v, int s, const sgh_laser* table, int n_steps, int step,
                               sgh_step_out* outs) {
  BState& st = v.st[s];
  st.table = table;
  st.outs = outs;
  st.n_steps = n_steps;
  st.step = step;
  st.active = step < n_steps ? 1 : 0;
  st.iters = 0;
  st.done = 1;
  st.iter = 0;
  st.pass1_ready = 0;
}

// ---------------------------------------------------------------------------
// step
// ---------------------------------------------------------------------------

__global__ void kb_run_setup(BView v, int n_steps) { v.g->steps_left = n_steps; }

// Laser state and Picard bookkeeping of every active slot; opens the loop.
__global__ void __launch_bounds__(CT) kb_begin(BView v, cudaGraphConditionalHandle h_picard, int in_graph) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < v.n; s += CT) {
    BState& st = v.st[s];
    const BSlot& sl = v.slot[s];
    if (st.active && st.step >= st.n_steps) st.active = 0;
    if (!st.active) {
      st.done = 1;
      continue;
    }
    st.laser = st.table[st.step];
    const sgh_laser L = st.laser;
    st.I0 = L.is_on ? sl.absorptivity * L.power / (sl.area_factor * (sl.r_x * sl.r_y)) : 0.0;
    const bool f32 = (L.flags & SGH_LASER_F32) != 0;
    st.shift_x = laser_shift(L.vx, sl.dt, sl.dx, f32);
    st.shift_y = laser_shift(L.vy, sl.dt, sl.dy, f32);
    st.iter = 0;
    st.status = SGH_STEP_CAPPED;
    st.rel_err = nan("");
    st.done = sl.max_iter > 0 ? 0 : 1;
    st.tickets = 0u;
    if (!st.done) atomicAdd(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v.g->picard_any = any > 0;
    v.g->n_iter_slots = any;
    v.g->slots_done = 0u;
    if (in_graph) cudaGraphSetConditional(h_picard, any > 0 ? 1u : 0u);
  }
}

// q_las, P_laser partials and q_net = q_las - shift(q_evap_old) per slot
// (solvers/spectral.py:273-306); q_net goes to the FP64 array (FP64 batches,
// q_net non-null) or to the xq operand plane (mixed precision).
//
// Each element's (y, x) is formed once and serves the flux, the shift and the
// operand plane. In mixed precision the point-sampled beam multiplies by the
// radii's reciprocals; the FP64 batch divides, in the reference's operation
// order, so that it tracks the single-instance plan to rounding. The register
// cap keeps
// three blocks per SM, so the FP64 arithmetic's fixed latencies are hidden by
// more warps.
__global__ void __launch_bounds__(BT, 3)
kb_face_begin(BView v, double* q_las, double* q_net, const double* q_evold, double* part_las) {
  // RB elements per block (RPT per thread, consecutive across the block per
  // round); the four shift taps of U elements are gathered before their use
  __shared__ double sh[2 * (BT / 32)];
  const int b = blockIdx.x;
  const int s = v.rblk_slot[b];
  const BSlot& sl = v.slot[s];
  const BState& st = v.st[s];
  if (!st.active) return;
  const int nx = sl.nx, ny = sl.ny;
  const double* f = q_evold + sl.face;
  const double I0 = st.I0, lx = st.laser.x, ly = st.laser.y, sx = st.shift_x, sy = st.shift_y;
  const double dx = sl.dx, dy = sl.dy, irx = 1.0 / sl.r_x, iry = 1.0 / sl.r_y, order = sl.order;
  const bool cell = sl.cell_integrated != 0, rcp = v.xq != nullptr;
  const int i0 = (b - sl.rblk0) * RB;
  double sum = 0.0, dummy = 0.0;
  constexpr int U = 2;
#pragma unroll 1
  for (int u0 = 0; u0 < RPT; u0 += U) {
    double g[U][4], wy0[U], wy1[U], wx0[U], wx1[U];
    bool ok[U], in[U];
    int ys[U], xs[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + (u0 + u) * BT + threadIdx.x;
      ok[u] = i < sl.S;
      const int y = ok[u] ? i / nx : 0, x = ok[u] ? i - y * nx : 0;
      ys[u] = y;
      xs[u] = x;
      const ShiftTap ty = shift_tap(y, ny, sy);
      const ShiftTap tx = shift_tap(x, nx, sx);
      in[u] = ok[u] && ty.in && tx.in;
      wy0[u] = ty.w0; wy1[u] = ty.w1; wx0[u] = tx.w0; wx1[u] = tx.w1;
      g[u][0] = in[u] ? f[ty.i0 * nx + tx.i0] : 0.0;
      g[u][1] = in[u] ? f[ty.i0 * nx + tx.i1] : 0.0;
      g[u][2] = in[u] ? f[ty.i1 * nx + tx.i0] : 0.0;
      g[u][3] = in[u] ? f[ty.i1 * nx + tx.i1] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + (u0 + u) * BT + threadIdx.x;
      double qn = 0.0;
      if (ok[u]) {
        const double xc = ((double)xs[u] + 0.5) * dx, yc = ((double)ys[u] + 0.5) * dy;
        double q;
        if (cell) {
          q = laser_flux(sl, I0, lx, ly, xc, yc);
        } else {  // point-sampled (super-)Gaussian (core/laser.py:42-53)
          const double ux = rcp ? (xc - lx) * irx : (xc - lx) / sl.r_x;
          const double uy = rcp ? (yc - ly) * iry : (yc - ly) / sl.r_y;
          const double r2 = ux * ux + uy * uy;
          q = I0 * ((order == 2.0) ? exp(-2.0 * r2) : exp(-2.0 * pow(r2, order / 2.0)));
        }
        q_las[sl.face + i] = q;
        sum += q;
        // the bilinear shift (spectral_cpu_kernels.py:328-371), zero outside the grid
        double val = wy0[u] * (wx0[u] * g[u][0] + wx1[u] * g[u][1]) + wy1[u] * (wx0[u] * g[u][2] + wx1[u] * g[u][3]);
        if (!in[u]) val = 0.0;
        qn = q - val;
        if (q_net) q_net[sl.face + i] = qn;
      }
      plane_put_yx(v.xq, sl, ys[u], xs[u], qn, ok[u]);
    }
  }
  block_sum2<BT>(sum, dummy, sh);
  if (threadIdx.x == 0) part_las[b] = sum;
}

// A = Zt + W_tt sigma (top-surface input of the current iterate).
__global__ void __launch_bounds__(BT)
kb_assemble(BView v, const double* Zt, const double* Wtt, const double* sigma, double* A) {
  const int b = blockIdx.x;
  const int s = v.blk_slot[b];
  const BSlot& sl = v.slot[s];
  if (!v.st[s].active) return;
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  double a = 0.0;
  if (i < sl.S) {
    a = Zt[sl.face + i] + Wtt[sl.face + i] * sigma[sl.face + i];
    A[sl.face + i] = a;
  }
  plane_put_block(v.xa, sl, i, a, i < sl.S);
}

// ---- batched face transform: one 2 x 4-register-tile block per tile ------
// DIR 0: x-pass out[y][k] = sum_n M[k][n] in[y][n]  (N = nx)
// DIR 1: y-pass out[k][x] = sum_n M[k][n] in[n][x]  (N = ny)
// Each slot has ceil(nx/64) * ceil(ny/32) tiles in both directions. INV
// selects M^T (inverse transform). Slots that are inactive -- or done, when
// SKIP_DONE -- are skipped. The tile body is axis_tile (sgh_axis.cuh).
template <class Epi>
struct SlotEpi {  // adapts a batched epilogue to axis_tile's (idx, k, b, v, r)
  static constexpr int kReduce = 0;
  const BSlot* sl;
  BState* st;
  Epi e;
  double* partials;
  __device__ __forceinline__ void operator()(int idx, int, int, double v, Red& r) const {
    e(*sl, *st, sl->face + idx, v, r);
  }
};

inline __host__ __device__ int face_tiles(int nx, int ny) { return ((nx + 63) / 64) * ((ny + 31) / 32); }

template <int DIR, bool INV, bool SKIP_DONE, class Epi>
__global__ void __launch_bounds__(AX_THREADS) kb_face_axis(BView v, const double* in, Epi epi, double* part_tile) {
  __shared__ double red[AX_THREADS / 32];
  const int b = blockIdx.x;
  const int s = v.tile_slot[b];
  const BSlot& sl = v.slot[s];
  BState& st = v.st[s];
  if (!st.active || (SKIP_DONE && st.done)) return;
  const int t = b - sl.tile0;
  const int nx = sl.nx, ny = sl.ny;
  const int N = DIR == 0 ? nx : ny;
  const int A = DIR == 0 ? ny : 1;
  const int Bs = DIR == 0 ? 1 : nx;
  constexpr int TK = DIR == 0 ? 64 : 32;
  constexpr int TC = DIR == 0 ? 32 : 64;
  const int ncx = (A * Bs + TC - 1) / TC;
  const int c0 = (t % ncx) * TC, k0 = (t / ncx) * TK;
  const double* M = v.mats + (DIR == 0 ? sl.mx : sl.my) + (INV ? (size_t)N * N : 0);
  Red r;
  SlotEpi<Epi> ad{&sl, &st, epi, nullptr};
  axis_tile<DIR == 0, 2, 4>(in + sl.face, M, N, N, A, Bs, c0, k0, ad, r);
  if (Epi::kMax) {
    double m = r.mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = red[0];
      for (int w = 1; w < AX_THREADS / 32; ++w) mm = fmax(mm, red[w]);
      part_tile[b] = mm;
    }
  }
}

// End of a Picard iteration's relaxation block (kb_relax, or kb_fy with the
// relaxation epilogue): publish the block's residual / iterate norm partials
// at part[2 p], part[2 p + 1] (p: the block's partial index; slot s has the
// np partials p0 .. p0 + np - 1) and take a ticket. The block drawing the slot's
// last ticket sums that slot's partials in a fixed order (so a slot's result
// does not depend on the rest of the batch) and runs its convergence test
// (solvers/spectral.py:464-499); the finisher of the last iterating slot sets
// the Picard loop condition and the number of slots that iterate next. No
// block waits on another. Called by every thread of the block.
template <int NT>
__device__ void relax_finish(const BView& v, int s, int p, int p0, int np, double r2, double o2, double* part,
                             const double* part_n1, cudaGraphConditionalHandle h_picard, int in_graph,
                             double* sh) {
  __shared__ unsigned ticket;
  __shared__ int last, count;
  const BSlot& sl = v.slot[s];
  BState& st = v.st[s];
  block_sum2<NT>(r2, o2, sh);
  if (threadIdx.x == 0) {
    part[2 * p] = r2;
    part[2 * p + 1] = o2;
    __threadfence();
    ticket = atomicAdd(&st.tickets, 1u);
  }
  __syncthreads();
  if (ticket != (unsigned)np - 1u) return;
  // this block finishes the slot
  __threadfence();
  double rs = 0.0, os = 0.0;
  for (int k = threadIdx.x; k < np; k += NT) {
    rs += __ldcg(part + 2 * (p0 + k));
    os += __ldcg(part + 2 * (p0 + k) + 1);
  }
  for (int k = threadIdx.x; k < sl.nblk; k += NT) os += __ldcg(part_n1 + sl.blk0 + k);
  block_sum2<NT>(rs, os, sh);
  if (threadIdx.x == 0) {
    const double n = sl.n_elements;
    const double rel = sqrt(rs / n) / fmax(sqrt(os / n), 1e-9);
    const int it = st.iter + 1;
    st.iter = it;
    st.rel_err = rel;
    if (rel < sl.tol) {
      st.status = SGH_STEP_CONVERGED;
      st.done = 1;
    } else if (!isfinite(rel)) {
      st.status = SGH_STEP_NONFINITE;
      st.done = 1;
    } else if (it >= sl.max_iter) {
      st.status = SGH_STEP_CAPPED;
      st.done = 1;
    }
    st.tickets = 0u;
    const int expect = __ldcg(&v.g->n_iter_slots);  // read before the ticket: the last finisher rewrites it
    __threadfence();
    last = atomicAdd(&v.g->slots_done, 1u) == (unsigned)expect - 1u;
    count = 0;
  }
  __syncthreads();
  if (!last) return;
  // the last finisher: slots iterating next, loop condition
  __threadfence();
  int c = 0;
  for (int k = threadIdx.x; k < v.n; k += NT)
    if (__ldcg(&v.st[k].active) && !__ldcg(&v.st[k].done)) ++c;
  if (c) atomicAdd(&count, c);
  __syncthreads();
  if (threadIdx.x == 0) {
    v.g->slots_done = 0u;
    v.g->n_iter_slots = count;
    v.g->picard_any = count > 0;
    if (in_graph) cudaGraphSetConditional(h_picard, count > 0 ? 1u : 0u);
  }
}

// ---- batched face transform on the tensor cores (mixed precision) ---------
// A 2-D transform of every slot's top face is two launches:
//   kb_fx   X1[y][c] = sum_x P[y][x] Mx[c][x]    (P: the slot's xa or xq plane)
//   kb_fy   G[r][c]  = sum_y My[r][y] X1[y][c], then the epilogue KIND
// Each CTA computes one 128-row x NB-column tile of one slot (MMA M = 128,
// N = NB). One thread streams the tile's operand chunks -- BF16 hi + lo, one
// bulk copy per operand and 32-slice chunk -- through a ring of f2::STAGES
// stages and issues three split-BF16 MMAs per 16-slice step (hi.hi, hi.lo,
// lo.hi) into one FP32 accumulator in tensor memory; the ring is primed
// before the tensor memory is allocated.
// kb_fx writes X1, split into BF16 hi + lo, to the slot's x1 plane, chunked
// and laid out exactly as the B operand chunks of kb_fy, which streams it
// like any other operand. Separability makes the tiles independent. A tile
// is a latency chain of nx/32 or ny/32 chunks, so the bytes the SM holds in
// flight decide the rate. Tiles of 128 columns take 32 KB per chunk where two
// 64-column tiles took 48 KB. Shared memory (2 stages of 32 KB) and tensor
// memory (one 128-column accumulator) allow three CTAs per SM, whose copies,
// MMAs and epilogues overlap. Measured against 64-column tiles at 2 x 4,
// 3 x 3 and 4 x 2 CTAs x stages, this is the fastest.
namespace f2 {
constexpr int THREADS = 256;
constexpr int NB = 128;                      // column block (MMA N)
constexpr int CA = umma::CHUNK_BYTES;        // 128 x 32 BF16 chunk of an A operand (8 KB)
constexpr int CBN = NB * umma::KC * 2;       // NB x 32 BF16 chunk of a B operand (8 KB)
// Column blocks per CTA: one A chunk could serve CB B chunks (CB = 2: 48 KB
// stages, two CTAs per SM), but at 288 serving slots that measured 3% slower
// than one block per CTA at three CTAs per SM (161.7K against 167.3K
// timesteps/s), so CB = 1.
constexpr int CB = 1;
constexpr int STAGE = 2 * CA + CB * 2 * CBN; // 32 KB: A hi/lo + CB x B hi/lo
constexpr int STAGES = 2;
constexpr int TAIL = 128;                    // barriers, TMEM address, status flag
constexpr int SMEM = STAGES * STAGE + TAIL;  // 65,664 bytes: three CTAs per SM
constexpr int CTAS = 3;                      // CTAs per SM (shared memory; CTAS x TCOLS <= 512)
constexpr uint32_t TCOLS = CB * NB;          // CB NB-column accumulators
static_assert(umma::TM * NB * 4 <= STAGES * STAGE, "the epilogue's FP32 tile fits in the drained ring");
static_assert(CTAS * TCOLS <= 512, "tensor memory of CTAS resident CTAs");
static_assert(CTAS * (SMEM + 1024) <= 228 * 1024, "shared memory of CTAS resident CTAs");
}  // namespace f2

// Tensor-core face tiles of a slot: 128-row tiles x groups of CB NB-column blocks.
inline __host__ __device__ int face_utiles(int nx, int ny) {
  const int ncb = (nx + f2::NB - 1) / f2::NB;
  return ((ncb + f2::CB - 1) / f2::CB) * ((ny + umma::TM - 1) / umma::TM);
}
// Bytes of a slot's x1 plane: NB-column blocks x 32-row chunks of {hi, lo}.
inline __host__ __device__ long long x1_bytes(int nx, int ny) {
  return (long long)((nx + f2::NB - 1) / f2::NB) * ((ny + umma::KC - 1) / umma::KC) * 2 * f2::CBN;
}

// Epilogue of the transform, on output element (r, c) of the slot's face:
//   F2_STORE    FP64 face array (x dct_scale if scaled)
//   F2_TOPFLUX  T_s -> evaporation -> q_evap (FP64, into the q_evap_old array), q_net -> xq plane
//   F2_COMMIT   T_temp and its block max
//   F2_SIGMA    sigma = dct_scale * G (FP64) and the first iterate's
//               A = Zt + W_tt sigma into the xa plane (replaces kb_assemble)
//   F2_RELAX    S_top = dct_scale * G straight into the Picard relaxation
//               (kb_relax's arithmetic: residual and iterate norms, sigma,
//               A = Zt + W_tt sigma into the xa plane), then the per-slot
//               convergence test (relax_finish); S_top is never stored
enum { F2_STORE = 0, F2_TOPFLUX = 1, F2_COMMIT = 2, F2_SIGMA = 3, F2_RELAX = 4 };

struct FaceParams {  // per-slot constants held in registers by the epilogues
  long long face, xa;
  int nx, ny;
  double recon_scale, dct_scale, T_liquidus, T_boil, evap_f1, evap_f2;
};

struct F2Args {
  double* out;        // F2_STORE target, F2_TOPFLUX q_evap (into the q_evap_old array), F2_COMMIT T_surf,
                      // F2_SIGMA and F2_RELAX sigma
  double* out2;       // unused
  const double* in2;  // F2_TOPFLUX q_las
  int scaled;
  const float* Zt;    // F2_SIGMA and F2_RELAX: the face sums and weights (FP32 in mixed batches)
  const float* Wtt;
  // F2_RELAX only
  const float* Yt;
  const float* Qtt;
  const double* part_n1;  // volume-pass norm partials
  double* part;           // relaxation partials, 2 per tile
  cudaGraphConditionalHandle h_picard;
  int in_graph;
};

// FP32 tile of 128 x NB results in shared memory: element (m, n) at
// m * NB + (n ^ (m & 31)) -- a column spreads over all banks for the TMEM
// copy, a row stays conflict-free for the epilogue.
__device__ __forceinline__ float f2_tile(const float* t, int m, int n) { return t[m * f2::NB + (n ^ (m & 31))]; }

// Shared-memory layout of both kernels: the ring, then full[STAGES],
// done[STAGES], the never-completed wait-test barrier, the TMEM address and
// the status flag.
struct F2Smem {
  char* ring;
  uint64_t *full, *done, *stall;
  uint32_t* tslot;
  volatile int* okflag;
  __device__ explicit F2Smem(char* sm)
      : ring(sm),
        full(reinterpret_cast<uint64_t*>(sm + f2::STAGES * f2::STAGE)),
        done(full + f2::STAGES),
        stall(done + f2::STAGES),
        tslot(reinterpret_cast<uint32_t*>(stall + 1)),
        okflag(reinterpret_cast<volatile int*>(tslot + 1)) {}
};

// Thread 0: initialise the barriers and issue the first min(n, STAGES)
// chunks; returns how many were issued.
template <class Load>
__device__ __forceinline__ int f2_prime(const F2Smem& m, int n, const Load& load) {
  using namespace umma;
  for (int i = 0; i < f2::STAGES; ++i) {
    mbar_init(&m.full[i], 1);
    mbar_init(&m.done[i], 1);
  }
  mbar_init(m.stall, 1);
  *m.okflag = 1;
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  const int pre = n < f2::STAGES ? n : f2::STAGES;
  for (int g = 0; g < pre; ++g) load(g);
  return pre;
}

// Thread 0: chunks 0..n-1 of the tile (chunk g in stage g % STAGES; each
// barrier completes one phase per use of its stage, so chunk g waits for
// parity (g / STAGES) & 1), MMAs into the accumulator at tmem, each stage
// refilled once its MMAs have drained, then the wait for the last MMAs. A wait that expires
// (after `lim` polls) records the error, clears the status flag and drains,
// with the full bound, every copy and MMA in flight; returns false then.
// stall: first wait on a barrier that nothing completes (the wait test).
template <class Load>
__device__ bool f2_run(const F2Smem& m, int n, int nb, int issued, const Load& load, uint32_t tmem, unsigned lim,
                       bool stall, int* err) {
  using namespace umma;
  constexpr int S = f2::STAGES, NB = f2::NB;
  const uint32_t idesc = idesc_bf16_f32(TM, NB);
  int committed = 0;
  bool ok = !stall || mbar_wait_bounded(m.stall, 0u, lim);
  for (int g = 0; g < n && ok; ++g) {
    if (!mbar_wait_bounded(&m.full[g % S], (uint32_t)((g / S) & 1), lim)) {
      ok = false;
      break;
    }
    tc_fence_after();
    const uint32_t ah = smem_u32(m.ring + (g % S) * f2::STAGE), al = ah + f2::CA;
#pragma unroll
    for (int k = 0; k < KC / 16; ++k) {
      const uint32_t oa = (uint32_t)(2 * k * (TM / 8) * 128), ob = (uint32_t)(2 * k * (NB / 8) * 128);
      const uint64_t dah = smem_desc(ah + oa, (TM / 8) * 128, 128);
      const uint64_t dal = smem_desc(al + oa, (TM / 8) * 128, 128);
      const uint32_t acc = (g > 0 || k > 0) ? 1u : 0u;
#pragma unroll
      for (int j = 0; j < f2::CB; ++j) {
        if (j < nb) {  // block j: B chunk at 2 CA + j 2 CBN, accumulator columns j NB..
          const uint32_t bh = ah + 2 * f2::CA + (uint32_t)(j * 2 * f2::CBN), bl = bh + f2::CBN;
          const uint64_t dbh = smem_desc(bh + ob, (NB / 8) * 128, 128);
          const uint64_t dbl = smem_desc(bl + ob, (NB / 8) * 128, 128);
          const uint32_t tj = tmem + (uint32_t)(j * NB);
          mma_bf16(tj, dah, dbh, idesc, acc);
          mma_bf16(tj, dah, dbl, idesc, 1u);
          mma_bf16(tj, dal, dbh, idesc, 1u);
        }
      }
    }
    mma_commit(&m.done[g % S]);
    committed = g + 1;
    // this stage takes chunk g + S as soon as its MMAs have drained (a few
    // hundred cycles, against the L2 latency of a chunk), so every stage of
    // the ring stays in flight
    const int nxt = g + S;
    if (nxt < n) {
      if (!mbar_wait_bounded(&m.done[g % S], (uint32_t)((g / S) & 1), lim)) {
        ok = false;
        break;
      }
      load(nxt);
      issued = nxt + 1;
    }
  }
  if (ok && n > 0) ok = mbar_wait_bounded(&m.done[(n - 1) % S], (uint32_t)(((n - 1) / S) & 1), lim);
  if (!ok) {
    atomicExch(err, 1);
    *m.okflag = 0;
    for (int g = issued - S < 0 ? 0 : issued - S; g < issued; ++g)
      mbar_wait_bounded(&m.full[g % S], (uint32_t)((g / S) & 1), WAIT_LIMIT);
    for (int g = committed - S < 0 ? 0 : committed - S; g < committed; ++g)
      mbar_wait_bounded(&m.done[g % S], (uint32_t)((g / S) & 1), WAIT_LIMIT);
  }
  return ok;
}

// 32 x 16 accumulator values of this warp's lane quarter.
__device__ __forceinline__ void f2_read16(uint32_t ta, float (&x)[16]) { umma::tmem_ld16(ta, x); }

template <bool INV, bool SKIP_DONE>
__global__ void __launch_bounds__(f2::THREADS, f2::CTAS) kb_fx(BView v) {
  using namespace umma;
  constexpr int CA = f2::CA, CBN = f2::CBN, NB = f2::NB;
  extern __shared__ __align__(128) char sm[];
  const int b = blockIdx.x;
  const int s = v.utile_slot[b];
  const BSlot& sl = v.slot[s];
  const BState& st = v.st[s];
  if (!st.active || (SKIP_DONE && st.done)) return;
  const int nx = sl.nx, ny = sl.ny;
  // tile t: row tile rt, column blocks cb0 .. cb0 + nb - 1
  const int ncb = (nx + NB - 1) / NB, ngb = (ncb + f2::CB - 1) / f2::CB;
  const int t = b - sl.utile0, rt = t / ngb, cb0 = (t - rt * ngb) * f2::CB, nb = min(f2::CB, ncb - cb0);
  const int nkx = (nx + KC - 1) / KC, nky = (ny + KC - 1) / KC;
  const F2Smem m(sm);
  const char* pp = (INV ? v.xa : v.xq) + sl.xa + (size_t)rt * nkx * 2 * CA;        // 128-row pair chunks
  const char* mx = v.mp + (INV ? sl.mpx_inv : sl.mpx) + (size_t)cb0 * nkx * 2 * CBN;  // 128-row pair chunks
  auto load = [&](int g) {  // P chunk (rt, g) and the Mx chunks (cb0 + j, g)
    char* stg = m.ring + (g % f2::STAGES) * f2::STAGE;
    uint64_t* bar = &m.full[g % f2::STAGES];
    mbar_expect_tx(bar, (uint32_t)(2 * CA + nb * 2 * CBN));
    bulk_g2s(stg, pp + (size_t)g * 2 * CA, 2 * CA, bar);
    for (int j = 0; j < nb; ++j)
      bulk_g2s(stg + 2 * CA + j * 2 * CBN, mx + ((size_t)j * nkx + g) * 2 * CBN, 2 * CBN, bar);
  };
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int issued = 0;
  if (tid == 0) issued = f2_prime(m, nkx, load);
  __syncwarp();
  if (warp == 0) tmem_alloc(m.tslot, f2::TCOLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *m.tslot;
  if (tid == 0) {
    const unsigned lim = v.g->wait_limit ? v.g->wait_limit : WAIT_LIMIT;
    f2_run(m, nkx, nb, issued, load, tmem, lim, false, &v.g->umma_err);
  }
  __syncthreads();
  if (*m.okflag) {
    // X1 row y = TMEM lane -> x1 plane element (row c, k = y); rows y and
    // y + 1 (lanes l, l + 1) go out as one 32-bit store per part
    tc_fence_after();
    const int q = warp & 3, half = warp >> 2;  // TMEM lane quarter, column half
    const int y = rt * TM + q * 32 + lane;
    const bool keep = y < nky * KC;
    const int c = half * (NB / 2);
#pragma unroll 1
    for (int jc = 0; jc < nb * (NB / 2); jc += 16) {
      const int j = jc / (NB / 2), cc = jc - j * (NB / 2);  // column block j, its columns c + cc ..
      char* x1 = v.x1 + sl.x1 + (size_t)(cb0 + j) * nky * 2 * CBN + (size_t)(y >> 5) * 2 * CBN;
      float x16[16];
      f2_read16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(j * NB + c + cc), x16);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        __nv_bfloat16 h, l;
        split_bf16((double)x16[i], h, l);
        const uint32_t hv = __bfloat16_as_ushort(h), lv = __bfloat16_as_ushort(l);
        const uint32_t hn = __shfl_down_sync(0xffffffffu, hv, 1);
        const uint32_t ln = __shfl_down_sync(0xffffffffu, lv, 1);
        if ((lane & 1) == 0 && keep) {
          const uint32_t o = core_off(c + cc + i, y & 31, NB);
          *reinterpret_cast<uint32_t*>(x1 + o) = hv | (hn << 16);
          *reinterpret_cast<uint32_t*>(x1 + CBN + o) = lv | (ln << 16);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, f2::TCOLS);
}

template <bool INV, bool SKIP_DONE, int KIND>
__global__ void __launch_bounds__(f2::THREADS, f2::CTAS) kb_fy(BView v, F2Args args, double* part_tile) {
  using namespace umma;
  constexpr int CA = f2::CA, CBN = f2::CBN, NB = f2::NB;
  extern __shared__ __align__(128) char sm[];
  __shared__ double red[2 * (f2::THREADS / 32)];
  const int b = blockIdx.x;
  const int s = v.utile_slot[b];
  const BSlot& sl = v.slot[s];
  const BState& st = v.st[s];
  if (!st.active || (SKIP_DONE && st.done)) return;
  FaceParams fp;
  fp.face = sl.face; fp.xa = sl.xa; fp.nx = sl.nx; fp.ny = sl.ny;
  fp.recon_scale = sl.recon_scale; fp.dct_scale = sl.dct_scale; fp.T_liquidus = sl.T_liquidus;
  fp.T_boil = sl.T_boil; fp.evap_f1 = sl.evap_f1; fp.evap_f2 = sl.evap_f2;
  const int nx = fp.nx, ny = fp.ny;
  // tile t: row tile rt, column blocks cb0 .. cb0 + nb - 1
  const int ncb = (nx + NB - 1) / NB, ngb = (ncb + f2::CB - 1) / f2::CB;
  const int t = b - sl.utile0, rt = t / ngb, cb0 = (t - rt * ngb) * f2::CB, nb = min(f2::CB, ncb - cb0);
  const int nkx = (nx + KC - 1) / KC, nky = (ny + KC - 1) / KC;
  const F2Smem m(sm);
  const char* my = v.mp + (INV ? sl.mpy_inv : sl.mpy) + (size_t)rt * nky * 2 * CA;  // 128-row pair chunks
  const char* x1 = v.x1 + sl.x1 + (size_t)cb0 * nky * 2 * CBN;                      // NB-row pair chunks
  auto load = [&](int g) {  // My chunk (rt, g) and the x1 chunks (cb0 + j, g)
    char* stg = m.ring + (g % f2::STAGES) * f2::STAGE;
    uint64_t* bar = &m.full[g % f2::STAGES];
    mbar_expect_tx(bar, (uint32_t)(2 * CA + nb * 2 * CBN));
    bulk_g2s(stg, my + (size_t)g * 2 * CA, 2 * CA, bar);
    for (int j = 0; j < nb; ++j)
      bulk_g2s(stg + 2 * CA + j * 2 * CBN, x1 + ((size_t)j * nky + g) * 2 * CBN, 2 * CBN, bar);
  };
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int issued = 0;
  if (tid == 0) issued = f2_prime(m, nky, load);
  __syncwarp();
  if (warp == 0) tmem_alloc(m.tslot, f2::TCOLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *m.tslot;
  if (tid == 0) {
    // the wait test: a wait that can only run out, with copies in flight
    const unsigned lim = v.g->wait_limit ? v.g->wait_limit : WAIT_LIMIT;
    f2_run(m, nky, nb, issued, load, tmem, lim, v.g->stall_test != 0, &v.g->umma_err);
  }
  __syncthreads();

  constexpr int ITEMS = TM * NB / f2::THREADS;  // tile elements per thread
  double mx = -INFINITY, r2 = 0.0, o2 = 0.0;
  const int r0 = rt * TM;
  float* tile = reinterpret_cast<float*>(m.ring);  // 128 x NB FP32 (64 KB) over the drained ring
  const bool good = *m.okflag != 0;
#pragma unroll 1
  for (int j = 0; j < nb; ++j) {  // column block cb0 + j: accumulator columns j NB ..
  const int c0 = (cb0 + j) * NB;
  if (good) {
    tc_fence_after();
    const int q = warp & 3, half = warp >> 2;
    const int mrow = q * 32 + lane;
    const int c = half * (NB / 2);
#pragma unroll 1
    for (int cc = 0; cc < NB / 2; cc += 16) {
      float x16[16];
      f2_read16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(j * NB + c + cc), x16);
#pragma unroll
      for (int i = 0; i < 16; ++i) tile[mrow * NB + ((c + cc + i) ^ (mrow & 31))] = x16[i];
    }
  }
  __syncthreads();
  if (good) {
    if (KIND == F2_TOPFLUX) {
      // a warp covers 32 consecutive x of one row (coalesced FP64 traffic);
      // the loads of U elements are issued ahead of their stores
      constexpr int U = 8;
      for (int it0 = 0; it0 < ITEMS; it0 += U) {
        double ql[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int y = r0 + e / NB, x = c0 + e % NB;
          ql[u] = (y < ny && x < nx) ? __ldg(args.in2 + fp.face + (long long)y * nx + x) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int mm = e / NB, n = e % NB;
          const int y = r0 + mm, x = c0 + n;
          const bool in = y < ny && x < nx;
          double qn = 0.0;
          if (in) {
            const double qe = evaporation(fp, fp.recon_scale * (double)f2_tile(tile, mm, n));
            args.out[fp.face + (long long)y * nx + x] = qe;
            qn = ql[u] - qe;
          }
          plane_put8_warp(v.xq + fp.xa, y, x, nkx, qn, in);
        }
      }
    } else if (KIND == F2_RELAX) {
      const double omega = sl.omega;
      constexpr int U = 4;
      for (int it0 = 0; it0 < ITEMS; it0 += U) {
        double sg[U], q[U], yt[U], zt[U], wt[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int y = r0 + e / NB, x = c0 + e % NB;
          const bool in = y < ny && x < nx;
          const long long j = fp.face + (long long)y * nx + x;
          sg[u] = in ? args.out[j] : 0.0;
          q[u] = in ? (double)__ldg(args.Qtt + j) : 0.0;
          yt[u] = in ? (double)__ldg(args.Yt + j) : 0.0;
          zt[u] = in ? (double)__ldg(args.Zt + j) : 0.0;
          wt[u] = in ? (double)__ldg(args.Wtt + j) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int mm = e / NB, n = e % NB;
          const int y = r0 + mm, x = c0 + n;
          const bool in = y < ny && x < nx;
          double a = 0.0;
          if (in) {  // kb_relax's update, with S_top from the tile
            const double d = fp.dct_scale * (double)f2_tile(tile, mm, n) - sg[u];
            r2 += d * d * q[u];
            o2 += 2.0 * sg[u] * yt[u] + sg[u] * sg[u] * q[u];
            const double ns = d * omega + sg[u];
            a = zt[u] + wt[u] * ns;
            args.out[fp.face + (long long)y * nx + x] = ns;
          }
          plane_put8_warp(v.xa + fp.xa, y, x, nkx, a, in);
        }
      }
    } else if (KIND == F2_SIGMA) {
      // 4 elements per round: at 8 the epilogue spilled at the 80-register
      // cap of three CTAs per SM, and the serving step measured 1.2% slower
      constexpr int U = 4;
      for (int it0 = 0; it0 < ITEMS; it0 += U) {
        double zt[U], wt[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int y = r0 + e / NB, x = c0 + e % NB;
          const bool in = y < ny && x < nx;
          const long long j = fp.face + (long long)y * nx + x;
          zt[u] = in ? (double)__ldg(args.Zt + j) : 0.0;
          wt[u] = in ? (double)__ldg(args.Wtt + j) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int mm = e / NB, n = e % NB;
          const int y = r0 + mm, x = c0 + n;
          const bool in = y < ny && x < nx;
          double a = 0.0;
          if (in) {
            const double sg = fp.dct_scale * (double)f2_tile(tile, mm, n);
            args.out[fp.face + (long long)y * nx + x] = sg;
            a = zt[u] + wt[u] * sg;
          }
          plane_put8_warp(v.xa + fp.xa, y, x, nkx, a, in);
        }
      }
    } else {
      constexpr int U = 4;
      for (int it0 = 0; it0 < ITEMS; it0 += U) {
        long long idx[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = tid + (it0 + u) * f2::THREADS;
          const int y = r0 + e / NB, x = c0 + e % NB;
          idx[u] = (y < ny && x < nx) ? fp.face + (long long)y * nx + x : -1;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (idx[u] < 0) continue;
          const int e = tid + (it0 + u) * f2::THREADS;
          const double val = (double)f2_tile(tile, e / NB, e % NB);
          if (KIND == F2_STORE) {
            args.out[idx[u]] = args.scaled ? val * fp.dct_scale : val;
          } else {  // F2_COMMIT
            const double T = fp.recon_scale * val;
            args.out[idx[u]] = T;
            mx = fmax(mx, T);
          }
        }
      }
    }
  }
  __syncthreads();  // every thread is done with the tile before the next block fills it
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, f2::TCOLS);
  if (KIND == F2_RELAX) {
    if (!good) r2 = nan("");  // a transform whose wait ran out ends the slot's step as non-finite
    relax_finish<f2::THREADS>(v, s, b, sl.utile0, sl.nutile, r2, o2, args.part, args.part_n1, args.h_picard,
                              args.in_graph, red);
  }
  if (KIND == F2_COMMIT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if (lane == 0) red[warp] = mx;
    __syncthreads();
    if (tid == 0) {
      double mm = red[0];
      for (int w = 1; w < f2::THREADS / 32; ++w) mm = fmax(mm, red[w]);
      part_tile[b] = mm;
    }
  }
}

struct EB_Store {  // out = v * (scaled ? dct_scale : 1)
  static constexpr int kMax = 0;
  double* out;
  int scaled;
  __device__ __forceinline__ void operator()(const BSlot& sl, const BState&, long long i, double v, Red&) const {
    out[i] = scaled ? v * sl.dct_scale : v;
  }
};

// The evaporation flux of the latest Picard iterate is written straight into
// the q_evap_old array: its one reader, the next step's warm-start shift in
// kb_face_begin, runs before this step's Picard loop, so the commit's copy
// q_evap_old <- q_evap (solvers/spectral.py:502-512) has nothing left to do.
struct EB_TopFlux {  // T_s -> evaporation -> q_net (solvers/spectral.py:388-404)
  static constexpr int kMax = 0;
  const double* q_las;
  double* q_ev;
  double* q_net;
  __device__ __forceinline__ void operator()(const BSlot& sl, const BState&, long long i, double v, Red&) const {
    const double Ts = sl.recon_scale * v;
    const double qe = evaporation(sl, Ts);
    q_ev[i] = qe;
    q_net[i] = q_las[i] - qe;
  }
};

struct EB_CommitSurface {  // T_temp and its max (solvers/spectral.py:502-512)
  static constexpr int kMax = 1;
  double* T_surf;
  __device__ __forceinline__ void operator()(const BSlot& sl, const BState&, long long i, double v, Red& r) const {
    const double T = sl.recon_scale * v;
    T_surf[i] = T;
    r.mx = fmax(r.mx, T);
  }
};

// Face-state update of one Picard iteration (see k_fs_relax in sgh_b200.cu):
// residual and iterate norms from the constant weights, relaxation of sigma
// and the next top-surface input A = Zt + W_tt sigma (FP64 array when A is
// given, xa operand plane in mixed precision); RPT elements per thread, loads
// ahead of stores. Then the per-slot convergence test
// (solvers/spectral.py:464-499) without a second launch: every block of a
// slot takes a ticket after publishing its partials; the block that draws the
// slot's last ticket sums that slot's partials in a fixed order (so a slot's
// result does not depend on the rest of the batch) and updates its state;
// the finisher of the last iterating slot sets the Picard loop condition and
// the number of slots that iterate next. No block waits on another.
__global__ void __launch_bounds__(BT)
kb_relax(BView v, const double* Zt, const double* Yt, const double* Wtt, const double* Qtt,
         const double* S_top, double* sigma, double* A, double* part, const double* part_n1,
         cudaGraphConditionalHandle h_picard, int in_graph) {
  __shared__ double sh[2 * (BT / 32)];
  const int b = blockIdx.x;
  const int s = v.rblk_slot[b];
  const BSlot& sl = v.slot[s];
  const BState& st = v.st[s];
  if (!st.active || st.done) return;
  const int i0 = (b - sl.rblk0) * RB;
  const long long face = sl.face;
  const double omega = sl.omega;
  double r2 = 0.0, o2 = 0.0;
  constexpr int U = 4;
#pragma unroll 1
  for (int u0 = 0; u0 < RPT; u0 += U) {
    double sg[U], q[U], yt[U], stp[U], zt[U], wt[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + (u0 + u) * BT + threadIdx.x;
      const bool ok = i < sl.S;
      const long long j = face + i;
      sg[u] = ok ? sigma[j] : 0.0;
      q[u] = ok ? __ldg(Qtt + j) : 0.0;
      yt[u] = ok ? __ldg(Yt + j) : 0.0;
      stp[u] = ok ? __ldg(S_top + j) : 0.0;
      zt[u] = ok ? __ldg(Zt + j) : 0.0;
      wt[u] = ok ? __ldg(Wtt + j) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + (u0 + u) * BT + threadIdx.x;
      const bool ok = i < sl.S;
      const double d = stp[u] - sg[u];
      r2 += d * d * q[u];
      o2 += 2.0 * sg[u] * yt[u] + sg[u] * sg[u] * q[u];
      const double ns = d * omega + sg[u];
      const double a = zt[u] + wt[u] * ns;
      if (ok) {
        sigma[face + i] = ns;
        if (A) A[face + i] = a;
      }
      plane_put_block(v.xa, sl, i, ok ? a : 0.0, ok);
    }
  }
  relax_finish<BT>(v, s, b, sl.rblk0, sl.nrblk, r2, o2, part, part_n1, h_picard, in_graph, sh);
}

// ---- volume passes ----------------------------------------------------------
// One thread per VEC consecutive (y, x) columns of a slot, looping over z;
// a, K and KK move as VEC-wide vectors (the slot's volume offset and face
// size are multiples of VEC). K comes from the K array or, when K is null,
// from the separable decay tables.
//   COMMIT = false: face sums of the propagated modes for the first step of a
//     slot: Zt = sum Ct K a, Yt = sum (K a) KK Ct, partials of sum (K a)^2
//     (later steps get them from the previous commit).
//   COMMIT = true: a = K a + KK Ct sigma (the modal commit), fused with the
//     same face sums for the next step, formed from the stored (type R) value
//     of a exactly as the first variant reads it back: the volume is read
//     once per step.
template <class R, int VEC>
struct VecOf { using T = R; };
template <>
struct VecOf<float, 4> { using T = float4; };
template <>
struct VecOf<float, 2> { using T = float2; };
template <>
struct VecOf<double, 2> { using T = double2; };

template <class R, int VEC>
__device__ __forceinline__ void vload(const R* p, R (&o)[VEC]) {
  using T = typename VecOf<R, VEC>::T;
  static_assert(sizeof(T) == VEC * sizeof(R), "no vector type of this width");
  const T t = *reinterpret_cast<const T*>(p);
#pragma unroll
  for (int c = 0; c < VEC; ++c) o[c] = reinterpret_cast<const R*>(&t)[c];
}
template <class R, int VEC>
__device__ __forceinline__ void vstore(R* p, const R (&o)[VEC]) {
  using T = typename VecOf<R, VEC>::T;
  static_assert(sizeof(T) == VEC * sizeof(R), "no vector type of this width");
  T t;
#pragma unroll
  for (int c = 0; c < VEC; ++c) reinterpret_cast<R*>(&t)[c] = o[c];
  *reinterpret_cast<T*>(p) = t;
}

// Mixed precision (FP32 modes): the volume pass works in FP32 registers,
// except the face sums and the norm. Per mode: K = Ex Ey Ez and KK (mode_kk)
// in FP32 from the FP64-derived 1-D tables, a <- K a + KK Ct sigma as two
// FP32 products and a fused add (relative rounding a few 1e-7, the order of
// the FP32 storage of a), and the face sums Zt, Yt and the norm partial
// gathered per column in FP32 over groups of VOL_FLUSH z-planes, each group's
// sum added in FP64 (a few 1e-7 relative, the order of the FP32 state). No
// FP64 arithmetic or conversion sits on the per-mode path, so the pass stays
// close to its 8 bytes per mode of HBM traffic. Every volume-pass variant
// groups the planes alike, so a slot's face sums do not depend on the vector
// width its batch runs at.
// FP64 modes: K and KK read from the volume arenas, everything in FP64.
template <class R, int VEC, bool COMMIT, int U>
__global__ void __launch_bounds__(BT / VEC, (sizeof(R) == 4 ? 3 : 2) * VEC)
kb_volume(BView v, R* a, const R* K, const R* KK, const double* sigma, R* Zt, R* Yt,
          double* part_n1) {
  constexpr bool TAB = sizeof(R) == 4;
  constexpr int NT = BT / VEC;
  __shared__ double sh[2 * (NT / 32)];
  const int b = blockIdx.x;
  const int s = v.blk_slot[b];
  const BSlot& sl = v.slot[s];
  BState& st = v.st[s];
  if (!st.active || (!COMMIT && st.pass1_ready)) return;
  const int i0 = (b - sl.blk0) * BT + VEC * threadIdx.x;
  double n1 = 0.0, dummy = 0.0;
  if (i0 < sl.S) {
    const double* ct = v.Ct + sl.zoff;
    const int nsum = sl.nx + sl.ny + sl.nz;
    const double* E = v.E + sl.eoff;
    const double* ez = E + sl.nx + sl.ny;
    const double* dz = ez + nsum;
    const double* lz = ez + 2 * nsum;
    const double dt_rc = sl.dt / (sl.rho * sl.cp);
    double zt[VEC], yt[VEC], sg[VEC];
    float zs[VEC], ys[VEC], ns[VEC];  // FP32 partial sums over VOL_FLUSH planes (FP32 modes)
    float sg32[VEC], exy32[VEC], dxy32[VEC], lxy32[VEC];
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      const int i = i0 + c;
      const int ix = i % sl.nx, iy = sl.nx + i / sl.nx;
      sg[c] = COMMIT ? sigma[sl.face + i] : 0.0;
      sg32[c] = (float)sg[c];
      exy32[c] = TAB ? (float)(E[ix] * E[iy]) : 0.0f;
      dxy32[c] = TAB ? (float)(E[nsum + ix] + E[ix] * E[nsum + iy]) : 0.0f;
      lxy32[c] = TAB ? (float)(E[2 * nsum + ix] + E[2 * nsum + iy]) : 0.0f;
      zt[c] = 0.0;
      yt[c] = 0.0;
      zs[c] = ys[c] = ns[c] = 0.0f;
    }
    // U planes per round: every load of the round is issued before its
    // arithmetic, so U x VEC values per thread are in flight
    for (int p0 = 0; p0 < sl.nz; p0 += U) {
      R av[U][VEC], kkv[U][VEC], kvv[U][VEC];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (p0 + u < sl.nz) {
          const long long j0 = sl.vol + (long long)(p0 + u) * sl.S + i0;
          vload<R, VEC>(a + j0, av[u]);
          if (!TAB) {
            vload<R, VEC>(KK + j0, kkv[u]);
            vload<R, VEC>(K + j0, kvv[u]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int p = p0 + u;
        if (p < sl.nz) {
          const double cp = ct[p];
          if (TAB) {
            const float cp32 = (float)cp, ez32 = (float)ez[p];
            const float dz32 = (float)dz[p], lz32 = (float)lz[p];
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
              const float kv = exy32[c] * ez32;
              const float num = fmaf(exy32[c], dz32, dxy32[c]);
              const float den = lxy32[c] + lz32;
              const float kk = den > 0.0f ? __fdividef(num, den) : (float)dt_rc;
              const float t = kk * cp32;
              float x = (float)av[u][c];
              if (COMMIT) x = fmaf(x, kv, t * sg32[c]);
              av[u][c] = (R)x;
              const float ak = x * kv;
              zs[c] = fmaf(cp32, ak, zs[c]);
              ys[c] = fmaf(ak, t, ys[c]);
              ns[c] = fmaf(ak, ak, ns[c]);
            }
            if ((p + 1) % VOL_FLUSH == 0 || p + 1 == sl.nz) {
#pragma unroll
              for (int c = 0; c < VEC; ++c) {
                zt[c] += (double)zs[c];
                yt[c] += (double)ys[c];
                n1 += (double)ns[c];
                zs[c] = ys[c] = ns[c] = 0.0f;
              }
            }
          } else {
#pragma unroll
            for (int c = 0; c < VEC; ++c) {
              const double kv = (double)kvv[u][c];
              const double kk = (double)kkv[u][c];
              if (COMMIT) av[u][c] = (R)((double)av[u][c] * kv + kk * (cp * sg[c]));
              const double ak = (double)av[u][c] * kv;
              zt[c] = fma(cp, ak, zt[c]);
              yt[c] = fma(ak * kk, cp, yt[c]);
              n1 = fma(ak, ak, n1);
            }
          }
          if (COMMIT) vstore<R, VEC>(a + sl.vol + (long long)p * sl.S + i0, av[u]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      Zt[sl.face + i0 + c] = (R)zt[c];
      Yt[sl.face + i0 + c] = (R)yt[c];
    }
  }
  block_sum2<NT>(n1, dummy, sh);
  if (threadIdx.x == 0) {
    part_n1[b] = n1;
    if (COMMIT) st.pass1_ready = 1;
  }
}

// Mixed-precision volume pass with a shared-memory ring. The block's BT face
// columns of each z-plane (FP32 modes: 1 KB, contiguous) arrive by one bulk
// copy per plane, completing on that stage's mbarrier, RING planes ahead of
// the arithmetic. The bytes in flight then come from shared memory, not from
// registers. Arithmetic and outputs are those of kb_volume's FP32 path (the
// face sums per column in FP32 over groups of VOL_FLUSH planes). A copy
// wait that expires sets the batch's error flag; the block then waits (with
// the full bound) for its copies in flight, writes a NaN norm partial so the
// Picard test stops, and leaves its face sums unwritten.
template <bool COMMIT, int RING>
__global__ void __launch_bounds__(BT / 4, 12)
kb_volume_ring(BView v, float* a, const double* sigma, float* Zt, float* Yt, double* part_n1) {
  constexpr int VEC = 4, NT = BT / VEC;
  static_assert(RING % 2 == 0, "planes are consumed two at a time");
  __shared__ __align__(128) float ring[RING][BT];
  __shared__ float ztab[4][RING_TABMAX];  // Ct, Ez, 1 - Ez, L_z of each plane in FP32 (nz <= RING_TABMAX)
  __shared__ uint64_t full[RING];
  __shared__ double sh[2 * (NT / 32)];
  __shared__ int bad;
  const int b = blockIdx.x;
  const int s = v.blk_slot[b];
  const BSlot& sl = v.slot[s];
  BState& st = v.st[s];
  if (!st.active || (!COMMIT && st.pass1_ready)) return;
  const int base = (b - sl.blk0) * BT;  // first face column of the block
  const int i0 = base + VEC * threadIdx.x;
  const int ncol = min(BT, sl.S - base);  // positive; a multiple of 4 (S is)
  const uint32_t bytes = (uint32_t)ncol * 4u;
  const int nz = sl.nz;
  float* col = a + sl.vol + base;  // plane p of the block at col + p * S (16-byte aligned)
  {
    const double* ct = v.Ct + sl.zoff;
    const int nsum = sl.nx + sl.ny + sl.nz;
    const double* ez = v.E + sl.eoff + sl.nx + sl.ny;
    for (int p = threadIdx.x; p < nz; p += NT) {  // the per-plane constants, converted once per block
      ztab[0][p] = (float)ct[p];
      ztab[1][p] = (float)ez[p];
      ztab[2][p] = (float)ez[nsum + p];
      ztab[3][p] = (float)ez[2 * nsum + p];
    }
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < RING; ++k) umma::mbar_init(&full[k], 1);
    bad = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    for (int p = 0; p < RING && p < nz; ++p) {
      umma::mbar_expect_tx(&full[p], bytes);
      umma::bulk_g2s(ring[p], col + (size_t)p * sl.S, bytes, &full[p]);
    }
  }
  __syncthreads();
  const bool live = i0 < sl.S;
  const float dt_rc = (float)(sl.dt / (sl.rho * sl.cp));
  double zt[VEC], yt[VEC], n1 = 0.0, dummy = 0.0;
  // FP32 partial sums over VOL_FLUSH planes, added into the FP64 sums at the
  // end of each group: three conversions per column and group instead of two
  // per mode (conversions and the quotient's reciprocal share the XU pipe)
  float zs[VEC], ys[VEC], ns[VEC];
  float sg32[VEC], exy32[VEC], dxy32[VEC], lxy32[VEC];
  {
    const double* E = v.E + sl.eoff;
    const int nsum = sl.nx + sl.ny + sl.nz;
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      const int i = live ? i0 + c : 0;
      const int ix = i % sl.nx, iy = sl.nx + i / sl.nx;
      sg32[c] = (COMMIT && live) ? (float)sigma[sl.face + i] : 0.0f;
      exy32[c] = (float)(E[ix] * E[iy]);
      dxy32[c] = (float)(E[nsum + ix] + E[ix] * E[nsum + iy]);
      lxy32[c] = (float)(E[2 * nsum + ix] + E[2 * nsum + iy]);
      zt[c] = 0.0;
      yt[c] = 0.0;
      zs[c] = ys[c] = ns[c] = 0.0f;
    }
  }
  // one z-plane of this thread's VEC columns (mode_kk's arithmetic, FP32)
  auto plane = [&](int p, const float* src) {
    const float cp32 = ztab[0][p], ez32 = ztab[1][p], dz32 = ztab[2][p], lz32 = ztab[3][p];
    const float4 x4 = *reinterpret_cast<const float4*>(src + VEC * threadIdx.x);
    float av[VEC] = {x4.x, x4.y, x4.z, x4.w};
    const bool zero_mode = (p | i0) == 0;  // column 0 (x = y = 0), plane 0: the quotient there is 0 / 0
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      float kk = __fdividef(fmaf(exy32[c], dz32, dxy32[c]), lxy32[c] + lz32);
      if (c == 0 && zero_mode) kk = dt_rc;  // KK of the zero mode
      const float kv = exy32[c] * ez32, t = kk * cp32;
      float x = av[c];
      if (COMMIT) x = fmaf(x, kv, t * sg32[c]);
      av[c] = x;
      const float ak = x * kv;
      zs[c] = fmaf(cp32, ak, zs[c]);
      ys[c] = fmaf(ak, t, ys[c]);
      ns[c] = fmaf(ak, ak, ns[c]);
    }
    if (COMMIT) *reinterpret_cast<float4*>(col + (size_t)p * sl.S + VEC * threadIdx.x) =
        make_float4(av[0], av[1], av[2], av[3]);
    if ((p + 1) % VOL_FLUSH == 0 || p + 1 == nz) {
#pragma unroll
      for (int c = 0; c < VEC; ++c) {
        zt[c] += (double)zs[c];
        yt[c] += (double)ys[c];
        n1 += (double)ns[c];
        zs[c] = ys[c] = ns[c] = 0.0f;
      }
    }
  };
  const unsigned lim = v.g->wait_limit ? v.g->wait_limit : umma::WAIT_LIMIT;
  // two planes per round (stages k and k + 1; RING is even): one barrier and
  // one refill round per two planes
  int p = 0;
  for (; p < nz; p += 2) {
    const int k = p % RING;
    const bool two = p + 1 < nz;
    bool arrived = umma::mbar_wait_bounded(&full[k], (uint32_t)((p / RING) & 1), lim);
    if (arrived && two) arrived = umma::mbar_wait_bounded(&full[k + 1], (uint32_t)((p / RING) & 1), lim);
    if (!arrived) bad = 1;
    if (arrived && live) {
      plane(p, ring[k]);
      if (two) plane(p + 1, ring[k + 1]);
    }
    __syncthreads();  // stages k, k + 1 are consumed by every thread; `bad` is visible
    if (bad) break;
    if (threadIdx.x == 0) {
      umma::fence_proxy_async();
      for (int q = 0; q < 2; ++q)
        if (p + q + RING < nz) {
          umma::mbar_expect_tx(&full[k + q], bytes);
          umma::bulk_g2s(ring[k + q], col + (size_t)(p + q + RING) * sl.S, bytes, &full[k + q]);
        }
    }
  }
  if (bad) {  // planes p .. min(nz, p + RING) - 1 were issued and not all consumed
    if (threadIdx.x == 0) {
      atomicExch(&v.g->umma_err, 1);
      for (int q = p; q < nz && q < p + RING; ++q)
        umma::mbar_wait_bounded(&full[q % RING], (uint32_t)((q / RING) & 1), umma::WAIT_LIMIT);
      part_n1[b] = nan("");
    }
    return;
  }
  if (live) {
#pragma unroll
    for (int c = 0; c < VEC; ++c) {
      Zt[sl.face + i0 + c] = (float)zt[c];
      Yt[sl.face + i0 + c] = (float)yt[c];
    }
  }
  block_sum2<NT>(n1, dummy, sh);
  if (threadIdx.x == 0) {
    part_n1[b] = n1;
    if (COMMIT) st.pass1_ready = 1;
  }
}

// Metrics of every active slot (solvers/spectral.py:536-542), one warp per
// slot; advances the step counters and decides whether the step loop goes on.
__global__ void __launch_bounds__(CT)
kb_commit(BView v, const double* part_las, const double* part_tile, int umma_tiles,
          cudaGraphConditionalHandle h_steps, int in_graph) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int s = warp; s < v.n; s += CT / 32) {
    BState& st = v.st[s];
    if (!st.active) continue;
    const BSlot& sl = v.slot[s];
    double p = 0.0, m = -INFINITY;
    for (int b = sl.rblk0 + lane; b < sl.rblk0 + sl.nrblk; b += 32) p += part_las[b];
    const int t0 = umma_tiles ? sl.utile0 : sl.tile0, nt = umma_tiles ? sl.nutile : sl.ntile;
    for (int b = t0 + lane; b < t0 + nt; b += 32) m = fmax(m, part_tile[b]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      p += __shfl_down_sync(0xffffffffu, p, o);
      m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    if (lane != 0) continue;
    sgh_step_out o;
    o.T_surface_max = m;
    o.P_laser = p * sl.dx * sl.dy;
    o.picard_rel_err = st.rel_err;
    o.n_iter = st.iter;
    o.converged = st.status == SGH_STEP_CONVERGED ? 1 : 0;
    o.status = st.status;
    o.flags = 0;
    st.last = o;
    if (st.outs) st.outs[st.step] = o;
    st.iters += st.iter;
    st.step += 1;
    if (st.step >= st.n_steps) st.active = 0;
    if (st.active) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int left = v.g->steps_left - 1;
    v.g->steps_left = left;
    if (in_graph) cudaGraphSetConditional(h_steps, (left > 0 && any) ? 1u : 0u);
  }
}

}  // namespace batch
}  // namespace sgh

using namespace sgh;
using namespace sgh::batch;

struct sgh_batch {
  int n = 0;
  int precision = 0;
  std::vector<sgh_config> cfg;
  std::vector<BSlot> slots;
  std::vector<int> blk_slot, rblk_slot, tile_slot, vblk_slot, utile_slot;  // block -> slot maps
  std::vector<std::pair<int, long long>> mat_list;  // (N, element offset)
  long long tot_vol = 0, tot_face = 0;
  int tot_blk = 0, tot_rblk = 0, tot_tile = 0, tot_vblk = 0, tot_z = 0, tot_utile = 0;
  long long mat_elems = 0;
  // workspace offsets (bytes)
  size_t o_slot, o_state, o_g, o_blk, o_rblk, o_tile, o_vblk, o_utile, o_mats, o_ct;
  size_t o_a, o_K, o_KK, o_E;
  long long tot_e = 0;
  size_t o_qlas, o_qnet, o_qevold, o_Stop, o_f1, o_sigma, o_A, o_Tsurf, o_Zt, o_Yt, o_Wtt, o_Qtt;
  size_t o_plas, o_pn1, o_prelax, o_ptile;
  size_t o_xa = 0, o_xq = 0, o_mp = 0, o_x1 = 0;  // operand pair planes (mixed)
  size_t xa_bytes = 0, mp_bytes = 0, x1_bytes = 0;
  int vec = 1;  // columns per thread of the volume passes
  int vol_unroll = 4;  // z-planes per load round of the volume passes (2, 4 or 8)
  std::vector<std::pair<int, long long>> mplane_list;  // (N, byte offset of the forward plane)
  size_t ws_need = 0;
  char* ws = nullptr;
  bool bound = false;
  int n_pre = 0, n_iter = 0, n_post = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cs1 = nullptr, cs2 = nullptr;

  size_t elem() const { return precision == SGH_PRECISION_MIXED ? sizeof(float) : sizeof(double); }
  double* d(size_t off) const { return reinterpret_cast<double*>(ws + off); }
  float* f(size_t off) const { return reinterpret_cast<float*>(ws + off); }
  BView view() const {
    BView v;
    v.slot = reinterpret_cast<const BSlot*>(ws + o_slot);
    v.st = reinterpret_cast<BState*>(ws + o_state);
    v.g = reinterpret_cast<BGlobal*>(ws + o_g);
    v.blk_slot = reinterpret_cast<const int*>(ws + o_blk);
    v.rblk_slot = reinterpret_cast<const int*>(ws + o_rblk);
    v.tile_slot = reinterpret_cast<const int*>(ws + o_tile);
    v.vblk_slot = reinterpret_cast<const int*>(ws + o_vblk);
    v.utile_slot = reinterpret_cast<const int*>(ws + o_utile);
    const bool mixed = precision == SGH_PRECISION_MIXED;
    v.xa = mixed ? ws + o_xa : nullptr;
    v.xq = mixed ? ws + o_xq : nullptr;
    v.x1 = mixed ? ws + o_x1 : nullptr;
    v.mp = mixed ? ws + o_mp : nullptr;
    v.mats = d(o_mats);
    v.Ct = d(o_ct);
    v.E = d(o_E);
    v.n = n;
    return v;
  }
};

namespace {

int bfail(int code, const std::string& m) { return sgh::set_error(code, m.c_str()); }

#define SGB_CK(call)                                                                        \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return bfail(SGH_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

inline int cdivl(long long a, long long b) { return (int)((a + b - 1) / b); }

thread_local int g_blaunch = 0;

// One 2-D transform of the top faces of all slots: the FP64 register-tiled
// contraction as an x-pass (in -> f1) and a y-pass (f1 -> epilogue ef), or,
// in mixed precision, the tensor-core x-pass of the xa (inverse) or xq
// (forward) operand plane into the x1 planes and the y-pass with epilogue KIND.
template <bool INV, bool SKIP, int KIND, class EpiF>
void face2d(sgh_batch* B, cudaStream_t s, const double* in, const EpiF& ef, const F2Args& fa, double* part) {
  const BView v = B->view();
  if (B->precision == SGH_PRECISION_MIXED) {
    (void)cudaFuncSetAttribute(kb_fx<INV, SKIP>, cudaFuncAttributeMaxDynamicSharedMemorySize, f2::SMEM);
    (void)cudaFuncSetAttribute(kb_fy<INV, SKIP, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, f2::SMEM);
    kb_fx<INV, SKIP><<<B->tot_utile, f2::THREADS, f2::SMEM, s>>>(v);
    kb_fy<INV, SKIP, KIND><<<B->tot_utile, f2::THREADS, f2::SMEM, s>>>(v, fa, part);
    g_blaunch += 2;
  } else {
    kb_face_axis<0, INV, SKIP, EB_Store><<<B->tot_tile, AX_THREADS, 0, s>>>(v, in, EB_Store{B->d(B->o_f1), 0},
                                                                            nullptr);
    kb_face_axis<1, INV, SKIP, EpiF><<<B->tot_tile, AX_THREADS, 0, s>>>(v, B->d(B->o_f1), ef, part);
    g_blaunch += 2;
  }
}

// One volume pass over all slots at the batch's vector width.
template <class R, bool COMMIT>
void launch_volume(sgh_batch* B, cudaStream_t s, R* a, const R* K, const R* KK) {
  const BView v = B->view();
  double *sg = B->d(B->o_sigma), *pn = B->d(B->o_pn1);
  R* zt = reinterpret_cast<R*>(B->ws + B->o_Zt);  // face sums in the modes' type
  R* yt = reinterpret_cast<R*>(B->ws + B->o_Yt);
  auto go = [&](auto vec, auto u) {
    constexpr int V_ = decltype(vec)::value, U_ = decltype(u)::value;
    kb_volume<R, V_, COMMIT, U_><<<B->tot_blk, BT / V_, 0, s>>>(v, a, K, KK, sg, zt, yt, pn);
  };
  auto with_u = [&](auto vec) {
    const int u = B->vol_unroll;
    if (u == 2) go(vec, std::integral_constant<int, 2>{});
    else if (u == 8) go(vec, std::integral_constant<int, 8>{});
    else go(vec, std::integral_constant<int, 4>{});
  };
  if constexpr (sizeof(R) == 4) {
    int max_nz = 0;
    for (const BSlot& sl : B->slots) max_nz = std::max(max_nz, sl.nz);
    if (B->vec == 4 && max_nz <= RING_TABMAX) {  // the ring form: 2 U planes of each block in flight
      float* af = reinterpret_cast<float*>(a);
      const int u = B->vol_unroll;
      if (u == 2) kb_volume_ring<COMMIT, 4><<<B->tot_blk, BT / 4, 0, s>>>(v, af, sg, zt, yt, pn);
      else if (u == 8) kb_volume_ring<COMMIT, 16><<<B->tot_blk, BT / 4, 0, s>>>(v, af, sg, zt, yt, pn);
      else kb_volume_ring<COMMIT, 8><<<B->tot_blk, BT / 4, 0, s>>>(v, af, sg, zt, yt, pn);
      return;
    }
  }
  if (B->vec >= 2) with_u(std::integral_constant<int, 2>{});  // vec 4 with nz > RING_TABMAX: float2
  else with_u(std::integral_constant<int, 1>{});
}

template <class R>
void enqueue_pre(sgh_batch* B, cudaStream_t s, cudaGraphConditionalHandle h, int in_graph) {
  const BView v = B->view();
  R* a = reinterpret_cast<R*>(B->ws + B->o_a);
  R* K = B->precision == SGH_PRECISION_MIXED ? nullptr : reinterpret_cast<R*>(B->ws + B->o_K);
  R* KK = B->precision == SGH_PRECISION_MIXED ? nullptr : reinterpret_cast<R*>(B->ws + B->o_KK);
  kb_begin<<<1, CT, 0, s>>>(v, h, in_graph);
  // mixed precision: q_net goes only into the operand plane of the transform
  kb_face_begin<<<B->tot_rblk, BT, 0, s>>>(v, B->d(B->o_qlas),
                                           B->precision == SGH_PRECISION_MIXED ? nullptr : B->d(B->o_qnet),
                                           B->d(B->o_qevold), B->d(B->o_plas));
  launch_volume<R, false>(B, s, a, K, KK);
  g_blaunch += 3;
  // initial guess: sigma = dct_scale * DCT2(q_las - shift(q_evap_old)), then A = Zt + W_tt sigma
  if (B->precision == SGH_PRECISION_MIXED) {
    face2d<false, false, F2_SIGMA>(B, s, B->d(B->o_qnet), EB_Store{B->d(B->o_sigma), 1},
                                   F2Args{B->d(B->o_sigma), nullptr, nullptr, 1, B->f(B->o_Zt), B->f(B->o_Wtt)},
                                   nullptr);
  } else {
    face2d<false, false, F2_STORE>(B, s, B->d(B->o_qnet), EB_Store{B->d(B->o_sigma), 1},
                                   F2Args{B->d(B->o_sigma), nullptr, nullptr, 1, nullptr}, nullptr);
    kb_assemble<<<B->tot_blk, BT, 0, s>>>(v, B->d(B->o_Zt), B->d(B->o_Wtt), B->d(B->o_sigma), B->d(B->o_A));
    g_blaunch += 1;
  }
}

void enqueue_picard(sgh_batch* B, cudaStream_t s, cudaGraphConditionalHandle h, int in_graph) {
  const BView v = B->view();
  const bool mixed = B->precision == SGH_PRECISION_MIXED;
  // T_s = IDCT2(A) -> evaporation -> q_net; S_top = dct_scale * DCT2(q_net)
  face2d<true, true, F2_TOPFLUX>(B, s, B->d(B->o_A), EB_TopFlux{B->d(B->o_qlas), B->d(B->o_qevold), B->d(B->o_qnet)},
                                 F2Args{B->d(B->o_qevold), nullptr, B->d(B->o_qlas), 0}, nullptr);
  if (mixed) {  // S_top straight into the relaxation and the convergence test (one launch less)
    F2Args fa{B->d(B->o_sigma), nullptr, nullptr, 1, B->f(B->o_Zt), B->f(B->o_Wtt), B->f(B->o_Yt), B->f(B->o_Qtt),
              B->d(B->o_pn1), B->d(B->o_prelax), h, in_graph};
    face2d<false, true, F2_RELAX>(B, s, B->d(B->o_qnet), EB_Store{B->d(B->o_Stop), 1}, fa, nullptr);
    return;
  }
  face2d<false, true, F2_STORE>(B, s, B->d(B->o_qnet), EB_Store{B->d(B->o_Stop), 1},
                                F2Args{B->d(B->o_Stop), nullptr, nullptr, 1}, nullptr);
  kb_relax<<<B->tot_rblk, BT, 0, s>>>(v, B->d(B->o_Zt), B->d(B->o_Yt), B->d(B->o_Wtt), B->d(B->o_Qtt),
                                     B->d(B->o_Stop), B->d(B->o_sigma), B->d(B->o_A),
                                     B->d(B->o_prelax), B->d(B->o_pn1), h, in_graph);
  g_blaunch += 1;
}

template <class R>
void enqueue_post(sgh_batch* B, cudaStream_t s, cudaGraphConditionalHandle h, int in_graph) {
  const BView v = B->view();
  R* a = reinterpret_cast<R*>(B->ws + B->o_a);
  R* K = B->precision == SGH_PRECISION_MIXED ? nullptr : reinterpret_cast<R*>(B->ws + B->o_K);
  R* KK = B->precision == SGH_PRECISION_MIXED ? nullptr : reinterpret_cast<R*>(B->ws + B->o_KK);
  face2d<true, false, F2_COMMIT>(B, s, B->d(B->o_A),
                                 EB_CommitSurface{B->d(B->o_Tsurf)},
                                 F2Args{B->d(B->o_Tsurf), nullptr, nullptr, 0}, B->d(B->o_ptile));
  launch_volume<R, true>(B, s, a, K, KK);
  kb_commit<<<1, CT, 0, s>>>(v, B->d(B->o_plas), B->d(B->o_ptile),
                             B->precision == SGH_PRECISION_MIXED ? 1 : 0, h, in_graph);
  g_blaunch += 2;
}

template <class R>
int capture(sgh_batch* B) {
  cudaGraph_t G;
  SGB_CK(cudaGraphCreate(&G, 0));
  B->graph = G;
  cudaGraphConditionalHandle h_steps;
  SGB_CK(cudaGraphConditionalHandleCreate(&h_steps, G, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams outer = {};
  outer.type = cudaGraphNodeTypeConditional;
  outer.conditional.handle = h_steps;
  outer.conditional.type = cudaGraphCondTypeWhile;
  outer.conditional.size = 1;
  cudaGraphNode_t outer_node;
  SGB_CK(cudaGraphAddNode(&outer_node, G, nullptr, 0, &outer));
  cudaGraph_t body = outer.conditional.phGraph_out[0];
  SGB_CK(cudaStreamBeginCaptureToGraph(B->cs1, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cudaGraphConditionalHandle h_picard;
  SGB_CK(cudaGraphConditionalHandleCreate(&h_picard, body, 0, 0));
  g_blaunch = 0;
  enqueue_pre<R>(B, B->cs1, h_picard, 1);
  B->n_pre = g_blaunch;
  cudaStreamCaptureStatus status;
  cudaGraph_t cur;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  SGB_CK(cudaStreamGetCaptureInfo(B->cs1, &status, nullptr, &cur, &deps, &ndeps));
  cudaGraphNodeParams inner = {};
  inner.type = cudaGraphNodeTypeConditional;
  inner.conditional.handle = h_picard;
  inner.conditional.type = cudaGraphCondTypeWhile;
  inner.conditional.size = 1;
  cudaGraphNode_t inner_node;
  SGB_CK(cudaGraphAddNode(&inner_node, cur, deps, ndeps, &inner));
  SGB_CK(cudaStreamUpdateCaptureDependencies(B->cs1, &inner_node, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t ibody = inner.conditional.phGraph_out[0];
  SGB_CK(cudaStreamBeginCaptureToGraph(B->cs2, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  g_blaunch = 0;
  enqueue_picard(B, B->cs2, h_picard, 1);
  B->n_iter = g_blaunch;
  SGB_CK(cudaStreamEndCapture(B->cs2, &ibody));
  g_blaunch = 0;
  enqueue_post<R>(B, B->cs1, h_steps, 1);
  B->n_post = g_blaunch;
  SGB_CK(cudaStreamEndCapture(B->cs1, &body));
  SGB_CK(cudaGetLastError());
  SGB_CK(cudaGraphInstantiate(&B->exec, G, 0));
  return SGH_OK;
}

struct LayoutB {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  }
};

}  // namespace

extern "C" {

int sgh_batch_create(const sgh_config* cfgs, int32_t n, int32_t precision, sgh_batch** out) {
  if (!cfgs || !out) return bfail(SGH_ERR_INVALID, "null argument");
  *out = nullptr;
  if (n < 1 || n > 65536) return bfail(SGH_ERR_INVALID, "slot count must be in [1, 65536]");
  if (precision != SGH_PRECISION_FP64 && precision != SGH_PRECISION_MIXED)
    return bfail(SGH_ERR_INVALID, "precision must be SGH_PRECISION_FP64 or SGH_PRECISION_MIXED");
  sgh_batch* B = new sgh_batch();
  B->n = n;
  B->precision = precision;
  B->cfg.assign(cfgs, cfgs + n);
  std::map<int, long long> mats;
  for (int i = 0; i < n; ++i) {
    const sgh_config& c = cfgs[i];
    std::string where = "slot " + std::to_string(i) + ": ";
    int rc = SGH_OK;
    if (c.nx < 2 || c.ny < 2 || c.nz < 2 || c.nx > 4096 || c.ny > 4096 || c.nz > 4096)
      rc = bfail(SGH_ERR_INVALID, where + "axis lengths must be in [2, 4096]");
    else if ((long long)c.nx * c.ny * c.nz > (1LL << 28))
      rc = bfail(SGH_ERR_INVALID, where + "grid exceeds 2^28 modes");
    else if (!(c.Lx > 0 && c.Ly > 0 && c.Lz > 0 && c.dt > 0 && c.r_x > 0 && c.r_y > 0 && c.area_factor > 0 &&
               c.order > 0))
      rc = bfail(SGH_ERR_INVALID, where + "sizes, dt, beam radii, order and area factor must be positive");
    else if (c.max_iter < 0 || c.max_iter > 1000000)
      rc = bfail(SGH_ERR_INVALID, where + "max_iter must be in [0, 1e6]");
    else if (c.cell_integrated && c.order != 2.0)
      rc = bfail(SGH_ERR_INVALID, where + "cell_integrated flux is only defined for the Gaussian");
    else if (c.box)
      rc = bfail(SGH_ERR_UNSUPPORTED, where + "box mode (fine_mesh) runs on single-instance plans only");
    else if (c.L_f > 0.0 || (c.has_model && !c.model_constant) || c.h_top > 0.0 || c.h_bottom > 0.0)
      rc = bfail(SGH_ERR_UNSUPPORTED,
                 where + "batches step the face-space form only (no latent heat, no T-dependent model, "
                         "no convection); use a single-instance plan");
    if (rc) {
      delete B;
      return rc;
    }
    mats[c.nx] = 0;
    mats[c.ny] = 0;
  }
  long long moff = 0;
  for (auto& kv : mats) {
    kv.second = moff;
    B->mat_list.push_back({kv.first, moff});
    moff += 2LL * kv.first * kv.first;
  }
  B->mat_elems = moff;
  std::map<int, long long> mplane;
  if (precision == SGH_PRECISION_MIXED) {
    long long po = 0;
    for (auto& kv : mats) {
      // per N: forward, inverse in 128-row chunks (the A operand of the
      // y-pass and the B operand of the x-pass alike)
      mplane[kv.first] = po;
      B->mplane_list.push_back({kv.first, po});
      po += 2LL * (long long)umma::pair_bytes<128>(kv.first, kv.first);
    }
    B->mp_bytes = (size_t)po;
  }
  for (int i = 0; i < n; ++i) {
    const sgh_config& c = cfgs[i];
    BSlot sl;
    std::memset(&sl, 0, sizeof(sl));
    sl.nx = c.nx; sl.ny = c.ny; sl.nz = c.nz;
    sl.S = c.nx * c.ny;
    sl.V = (long long)sl.S * c.nz;
    sl.max_iter = c.max_iter;
    sl.cell_integrated = c.cell_integrated;
    sl.vol = (B->tot_vol + 3) / 4 * 4;  // aligned for the vector volume passes
    sl.face = B->tot_face;
    sl.zoff = B->tot_z;
    sl.eoff = (int)B->tot_e;
    sl.mx = (int)mats[c.nx];
    sl.my = (int)mats[c.ny];
    sl.nblk = cdivl(sl.S, BT);
    sl.rblk0 = B->tot_rblk;
    sl.nrblk = cdivl(sl.S, RB);
    sl.ntile = face_tiles(c.nx, c.ny);
    sl.vblk0 = B->tot_vblk;
    sl.nvblk = cdivl(sl.V, BT);
    sl.nutile = face_utiles(c.nx, c.ny);
    if (precision == SGH_PRECISION_MIXED) {
      sl.xa = (long long)B->xa_bytes;
      B->xa_bytes += umma::pair_bytes<128>(c.ny, c.nx);
      sl.x1 = (long long)B->x1_bytes;
      B->x1_bytes += x1_bytes(c.nx, c.ny);
      sl.mpx = mplane[c.nx];
      sl.mpx_inv = sl.mpx + (long long)umma::pair_bytes<128>(c.nx, c.nx);
      sl.mpy = mplane[c.ny];
      sl.mpy_inv = sl.mpy + (long long)umma::pair_bytes<128>(c.ny, c.ny);
    }
    sl.Lx = c.Lx; sl.Ly = c.Ly; sl.Lz = c.Lz;
    sl.dx = c.Lx / c.nx; sl.dy = c.Ly / c.ny;
    sl.dt = c.dt;
    const double dz = c.Lz / c.nz;
    (void)dz;
    sl.dct_scale = (sl.dx * sl.dy) * std::sqrt((double)(c.nx * c.ny) / (c.Lx * c.Ly));
    sl.recon_scale = std::sqrt((double)(c.nx * c.ny)) / std::sqrt(c.Lx * c.Ly);
    sl.n_elements = (double)sl.V;
    sl.T0 = c.T0;
    sl.evap_f1 = 0.82 * c.dH_LV * c.Pa / std::sqrt(2 * M_PI * c.R_v);
    sl.evap_f2 = c.dH_LV / (c.R_v * c.T_boil);
    sl.T_boil = c.T_boil;
    sl.T_liquidus = c.T_liquidus;
    sl.r_x = c.r_x; sl.r_y = c.r_y;
    sl.absorptivity = c.absorptivity;
    sl.order = c.order;
    sl.area_factor = c.area_factor;
    sl.omega = c.omega;
    sl.tol = c.tol;
    sl.k = c.k; sl.rho = c.rho; sl.cp = c.cp;
    B->slots.push_back(sl);
    B->tot_vol = sl.vol + sl.V;
    B->tot_face += sl.S;
    B->tot_z += c.nz;
    B->tot_e += 3 * (c.nx + c.ny + c.nz);  // E, 1 - E and kbar k^2 per axis
    B->tot_rblk += sl.nrblk;
    B->tot_vblk += sl.nvblk;
    B->rblk_slot.insert(B->rblk_slot.end(), sl.nrblk, i);
    B->vblk_slot.insert(B->vblk_slot.end(), sl.nvblk, i);
  }
  // Column blocks and face tiles: the slots with the longest blocks take the
  // first block indices of a launch (a column block runs over nz planes, a face
  // tile over nx / 32 or ny / 32 chunks), so that a launch's last wave holds
  // its shortest blocks. Every slot keeps one contiguous range, and per-slot
  // partials are summed over it in a fixed order: a slot's results do not
  // depend on this order.
  {
    std::vector<int> by_z(n), by_face(n);
    for (int i = 0; i < n; ++i) by_z[i] = by_face[i] = i;
    const std::vector<BSlot>& S = B->slots;
    std::stable_sort(by_z.begin(), by_z.end(), [&](int a, int b) { return S[a].nz > S[b].nz; });
    std::stable_sort(by_face.begin(), by_face.end(), [&](int a, int b) {
      return S[a].nx != S[b].nx ? S[a].nx > S[b].nx : S[a].ny > S[b].ny;
    });
    for (int i : by_z) {
      BSlot& sl = B->slots[i];
      sl.blk0 = B->tot_blk;
      B->tot_blk += sl.nblk;
      B->blk_slot.insert(B->blk_slot.end(), sl.nblk, i);
    }
    for (int i : by_face) {
      BSlot& sl = B->slots[i];
      sl.tile0 = B->tot_tile;
      sl.utile0 = B->tot_utile;
      B->tot_tile += sl.ntile;
      B->tot_utile += sl.nutile;
      B->tile_slot.insert(B->tile_slot.end(), sl.ntile, i);
      B->utile_slot.insert(B->utile_slot.end(), sl.nutile, i);
    }
  }
  {
    const int vw = precision == SGH_PRECISION_MIXED ? 4 : 2;
    bool ok = true;
    for (const BSlot& sl : B->slots) ok = ok && (sl.S % vw == 0);
    B->vec = ok ? vw : 1;
  }
  LayoutB L;
  const size_t F8 = sizeof(double) * (size_t)B->tot_face;
  const size_t VE = B->elem() * (size_t)B->tot_vol;
  B->o_slot = L.take(sizeof(BSlot) * n);
  B->o_state = L.take(sizeof(BState) * n);
  B->o_g = L.take(sizeof(BGlobal));
  B->o_blk = L.take(sizeof(int) * (size_t)B->tot_blk);
  B->o_rblk = L.take(sizeof(int) * (size_t)B->tot_rblk);
  B->o_tile = L.take(sizeof(int) * (size_t)B->tot_tile);
  B->o_vblk = L.take(sizeof(int) * (size_t)B->tot_vblk);
  B->o_utile = L.take(sizeof(int) * (size_t)B->tot_utile);
  B->o_mats = L.take(sizeof(double) * (size_t)B->mat_elems);
  B->o_ct = L.take(sizeof(double) * (size_t)B->tot_z);
  B->o_a = L.take(VE);
  B->o_K = L.take(precision == SGH_PRECISION_MIXED ? 0 : VE);  // mixed: K from the decay tables
  B->o_KK = L.take(precision == SGH_PRECISION_MIXED ? 0 : VE);  // mixed: KK from the 1-D tables
  B->o_E = L.take(sizeof(double) * (size_t)B->tot_e);
  B->o_qlas = L.take(F8);
  B->o_qnet = L.take(precision == SGH_PRECISION_MIXED ? 0 : F8);  // mixed: the xq operand plane only
  B->o_qevold = L.take(F8);
  B->o_Stop = L.take(precision == SGH_PRECISION_MIXED ? 0 : F8);  // mixed: S_top stays in the transform
  B->o_f1 = L.take(precision == SGH_PRECISION_MIXED ? 0 : F8);  // the FP64 transforms' intermediate
  B->o_sigma = L.take(F8);
  B->o_A = L.take(precision == SGH_PRECISION_MIXED ? 0 : F8);  // mixed: A only as the xa operand plane
  B->o_Tsurf = L.take(F8);
  // face sums and weights in the modes' type: FP32 in mixed batches (their
  // rounding, 6e-8 relative, sits far below the BF16 split of the transform
  // operands they feed), FP64 otherwise
  const size_t FR = precision == SGH_PRECISION_MIXED ? sizeof(float) * (size_t)B->tot_face : F8;
  B->o_Zt = L.take(FR);
  B->o_Yt = L.take(FR);
  B->o_Wtt = L.take(FR);
  B->o_Qtt = L.take(FR);
  B->o_plas = L.take(sizeof(double) * B->tot_blk);
  B->o_pn1 = L.take(sizeof(double) * B->tot_blk);
  B->o_prelax = L.take(sizeof(double) * 2 * std::max(B->tot_rblk, B->tot_utile));  // per relaxation block or tile
  B->o_ptile = L.take(sizeof(double) * std::max(B->tot_tile, B->tot_utile));
  if (precision == SGH_PRECISION_MIXED) {
    B->o_xa = L.take(B->xa_bytes);
    B->o_xq = L.take(B->xa_bytes);
    B->o_mp = L.take(B->mp_bytes);
    B->o_x1 = L.take(B->x1_bytes);
  }
  B->ws_need = L.off;
  *out = B;
  return SGH_OK;
}

int sgh_batch_destroy(sgh_batch* B) {
  if (!B) return SGH_OK;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->cs1) cudaStreamDestroy(B->cs1);
  if (B->cs2) cudaStreamDestroy(B->cs2);
  delete B;
  return SGH_OK;
}

int sgh_batch_set_policy(sgh_batch* B, const sgh_batch_policy* pol) {
  if (!B || !pol) return bfail(SGH_ERR_INVALID, "null argument");
  if (B->bound) return bfail(SGH_ERR_STATE, "set the policy before sgh_batch_bind (the graphs are captured there)");
  const int u = pol->vol_unroll ? pol->vol_unroll : 4;
  if (u != 2 && u != 4 && u != 8) return bfail(SGH_ERR_INVALID, "vol_unroll must be 2, 4 or 8");
  const int vmax = B->precision == SGH_PRECISION_MIXED ? 4 : 2;
  const int vw = pol->vol_vec ? pol->vol_vec : vmax;
  if (vw != 1 && vw != 2 && vw != 4) return bfail(SGH_ERR_INVALID, "vol_vec must be 1, 2 or 4");
  if (vw > vmax) return bfail(SGH_ERR_INVALID, "vol_vec 4 needs FP32 modes (mixed precision)");
  for (int i = 0; i < 6; ++i)
    if (pol->reserved[i]) return bfail(SGH_ERR_INVALID, "reserved policy fields must be 0");
  bool ok = true;  // every slot's face a multiple of the vector width (offsets are padded to 4)
  for (const BSlot& sl : B->slots) ok = ok && (sl.S % vw == 0);
  B->vol_unroll = u;
  B->vec = ok ? vw : 1;
  return SGH_OK;
}

int sgh_batch_workspace_bytes(const sgh_batch* B, uint64_t* bytes) {
  if (!B || !bytes) return bfail(SGH_ERR_INVALID, "null argument");
  *bytes = B->ws_need;
  return SGH_OK;
}

int sgh_batch_bind(sgh_batch* B, void* workspace, uint64_t bytes, void* stream) {
  if (!B || !workspace) return bfail(SGH_ERR_INVALID, "null argument");
  if (B->bound) return bfail(SGH_ERR_STATE, "batch is already bound");
  if (bytes < B->ws_need) return bfail(SGH_ERR_WORKSPACE, "workspace is smaller than sgh_batch_workspace_bytes()");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return bfail(SGH_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  B->ws = static_cast<char*>(workspace);
  const int n = B->n;
  SGB_CK(cudaMemcpyAsync(B->ws + B->o_slot, B->slots.data(), sizeof(BSlot) * n, cudaMemcpyHostToDevice, s));
  SGB_CK(cudaMemsetAsync(B->ws + B->o_state, 0, sizeof(BState) * n, s));
  SGB_CK(cudaMemsetAsync(B->ws + B->o_g, 0, sizeof(BGlobal), s));
  const auto put = [&](size_t off, const std::vector<int>& m) {
    return cudaMemcpyAsync(B->ws + off, m.data(), sizeof(int) * m.size(), cudaMemcpyHostToDevice, s);
  };
  SGB_CK(put(B->o_blk, B->blk_slot));
  SGB_CK(put(B->o_rblk, B->rblk_slot));
  SGB_CK(put(B->o_tile, B->tile_slot));
  SGB_CK(put(B->o_vblk, B->vblk_slot));
  SGB_CK(put(B->o_utile, B->utile_slot));
  SGB_CK(cudaMemsetAsync(B->ws + B->o_qevold, 0, sizeof(double) * B->tot_face, s));
  for (auto& m : B->mat_list)
    kb_dct_matrix<<<cdivl((long long)m.first * m.first, BT), BT, 0, s>>>(m.first, B->d(B->o_mats) + m.second);
  const BView v = B->view();
  if (B->precision == SGH_PRECISION_MIXED) {
    SGB_CK(cudaMemsetAsync(B->ws + B->o_xa, 0, B->xa_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_xq, 0, B->xa_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_mp, 0, B->mp_bytes, s));
    for (size_t j = 0; j < B->mplane_list.size(); ++j) {
      const int N = B->mplane_list[j].first;
      const long long po = B->mplane_list[j].second;
      long long moff = -1;
      for (auto& m : B->mat_list)
        if (m.first == N) moff = m.second;
      const size_t pb = umma::pair_bytes<128>(N, N);
      auto pl = [&](size_t o) { return B->ws + B->o_mp + po + o; };
      const int g = cdivl((long long)N * N, BT);
      for (int inv = 0; inv < 2; ++inv) {
        kb_matrix_planes<128><<<g, BT, 0, s>>>(N, B->d(B->o_mats) + moff, inv, pl(inv * pb));
      }
    }
    kb_tables<float><<<B->tot_vblk, BT, 0, s>>>(v, nullptr, nullptr, B->d(B->o_ct), B->d(B->o_E));
    kb_weights<float><<<B->tot_blk, BT, 0, s>>>(v, nullptr, B->f(B->o_Wtt), B->f(B->o_Qtt));
  } else {
    double* K = B->d(B->o_K);
    double* KK = B->d(B->o_KK);
    kb_tables<double><<<B->tot_vblk, BT, 0, s>>>(v, K, KK, B->d(B->o_ct), B->d(B->o_E));
    kb_weights<double><<<B->tot_blk, BT, 0, s>>>(v, KK, B->d(B->o_Wtt), B->d(B->o_Qtt));
  }
  SGB_CK(cudaGetLastError());
  SGB_CK(cudaStreamSynchronize(s));
  SGB_CK(cudaStreamCreateWithFlags(&B->cs1, cudaStreamNonBlocking));
  SGB_CK(cudaStreamCreateWithFlags(&B->cs2, cudaStreamNonBlocking));
  const int rc = B->precision == SGH_PRECISION_MIXED ? capture<float>(B) : capture<double>(B);
  if (rc) return rc;
  B->bound = true;
  return SGH_OK;
}

int sgh_batch_slot_start(sgh_batch* B, int32_t slot, const sgh_laser* lasers_dev, int32_t n_steps,
                         sgh_step_out* outs_dev, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  if (slot < 0 || slot >= B->n) return bfail(SGH_ERR_INVALID, "slot out of range");
  if (n_steps < 0 || (n_steps > 0 && !lasers_dev)) return bfail(SGH_ERR_INVALID, "bad laser table");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const BSlot& sl = B->slots[slot];
  const int g = cdivl(std::max<long long>(sl.V, sl.S), BT);
  if (B->precision == SGH_PRECISION_MIXED)
    kb_slot_start<float><<<g, BT, 0, s>>>(B->view(), slot, reinterpret_cast<float*>(B->ws + B->o_a),
                                          B->d(B->o_qevold), B->d(B->o_sigma), lasers_dev,
                                          n_steps, outs_dev);
  else
    kb_slot_start<double><<<g, BT, 0, s>>>(B->view(), slot, B->d(B->o_a), B->d(B->o_qevold), B->d(B->o_sigma),
                                           lasers_dev, n_steps, outs_dev);
  SGB_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_batch_slot_resume(sgh_batch* B, int32_t slot, const sgh_laser* lasers_dev, int32_t n_steps,
                          int32_t step, sgh_step_out* outs_dev, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  if (slot < 0 || slot >= B->n) return bfail(SGH_ERR_INVALID, "slot out of range");
  if (n_steps < 0 || (n_steps > 0 && !lasers_dev)) return bfail(SGH_ERR_INVALID, "bad laser table");
  if (step < 0 || step > n_steps) return bfail(SGH_ERR_INVALID, "step must be in [0, n_steps]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  kb_slot_resume<<<1, 1, 0, s>>>(B->view(), slot, lasers_dev, n_steps, step, outs_dev);
  SGB_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_batch_slot_stop(sgh_batch* B, int32_t slot, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  if (slot < 0 || slot >= B->n) return bfail(SGH_ERR_INVALID, "slot out of range");
  kb_slot_stop<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(B->view(), slot);
  SGB_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_batch_step(sgh_batch* B, int32_t n_steps, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  if (n_steps < 0) return bfail(SGH_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return SGH_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  kb_run_setup<<<1, 1, 0, s>>>(B->view(), n_steps);
  SGB_CK(cudaGetLastError());
  SGB_CK(cudaGraphLaunch(B->exec, s));
  return SGH_OK;
}

int sgh_batch_step_eager(sgh_batch* B, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  kb_run_setup<<<1, 1, 0, s>>>(B->view(), 1);
  const bool mixed = B->precision == SGH_PRECISION_MIXED;
  if (mixed) enqueue_pre<float>(B, s, 0, 0);
  else enqueue_pre<double>(B, s, 0, 0);
  for (int it = 0; it < 1000000; ++it) {
    BGlobal g;
    SGB_CK(cudaMemcpyAsync(&g, B->ws + B->o_g, sizeof(BGlobal), cudaMemcpyDeviceToHost, s));
    SGB_CK(cudaStreamSynchronize(s));
    if (!g.picard_any) break;
    enqueue_picard(B, s, 0, 0);
  }
  if (mixed) enqueue_post<float>(B, s, 0, 0);
  else enqueue_post<double>(B, s, 0, 0);
  SGB_CK(cudaGetLastError());
  SGB_CK(cudaStreamSynchronize(s));
  return SGH_OK;
}

int sgh_batch_status(const sgh_batch* B, sgh_batch_slot_info* out, void* stream) {
  if (!B || !B->bound || !out) return bfail(SGH_ERR_INVALID, "batch not bound or null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<BState> st(B->n);
  SGB_CK(cudaMemcpyAsync(st.data(), B->ws + B->o_state, sizeof(BState) * B->n, cudaMemcpyDeviceToHost, s));
  SGB_CK(cudaStreamSynchronize(s));
  for (int i = 0; i < B->n; ++i) {
    out[i].active = st[i].active;
    out[i].step = st[i].step;
    out[i].n_steps = st[i].n_steps;
    out[i].iters = st[i].iters;
    out[i].last = st[i].last;
  }
  return SGH_OK;
}

int sgh_batch_buffer(const sgh_batch* B, int32_t slot, int32_t which, void** ptr, uint64_t* bytes) {
  if (!B || !ptr) return bfail(SGH_ERR_INVALID, "null argument");
  if (!B->ws) return bfail(SGH_ERR_STATE, "batch is not bound");
  if (slot < 0 || slot >= B->n) return bfail(SGH_ERR_INVALID, "slot out of range");
  const BSlot& sl = B->slots[slot];
  const size_t e = B->elem();
  size_t off, nb;
  switch (which) {
    case SGH_BUF_MODES: off = B->o_a + e * sl.vol; nb = e * sl.V; break;
    case SGH_BUF_K:
      if (B->precision == SGH_PRECISION_MIXED)
        return bfail(SGH_ERR_INVALID, "mixed-precision batches do not store K (it is formed from 1-D tables)");
      off = B->o_K + e * sl.vol;
      nb = e * sl.V;
      break;
    case SGH_BUF_KK:
      if (B->precision == SGH_PRECISION_MIXED)
        return bfail(SGH_ERR_INVALID, "mixed-precision batches do not store KK (it is formed from 1-D tables)");
      off = B->o_KK + e * sl.vol;
      nb = e * sl.V;
      break;
    case SGH_BUF_Q_EVAP_OLD: off = B->o_qevold + sizeof(double) * sl.face; nb = sizeof(double) * sl.S; break;
    case SGH_BUF_SURFACE: off = B->o_Tsurf + sizeof(double) * sl.face; nb = sizeof(double) * sl.S; break;
    default: return bfail(SGH_ERR_INVALID, "buffer id not available for batch slots");
  }
  *ptr = B->ws + off;
  if (bytes) *bytes = nb;
  return SGH_OK;
}

int sgh_batch_error(const sgh_batch* B, int32_t* err, void* stream) {
  if (!B || !B->bound || !err) return bfail(SGH_ERR_INVALID, "batch not bound or null output");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BGlobal g;
  SGB_CK(cudaMemcpyAsync(&g, B->ws + B->o_g, sizeof(BGlobal), cudaMemcpyDeviceToHost, s));
  SGB_CK(cudaStreamSynchronize(s));
  *err = g.umma_err;
  return SGH_OK;
}

int sgh_batch_set_wait_limit(sgh_batch* B, uint32_t polls, int32_t stall_test, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  if (stall_test && polls == 0) return bfail(SGH_ERR_INVALID, "the wait test needs an explicit poll bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned v[2] = {polls, stall_test ? 1u : 0u};
  static_assert(offsetof(BGlobal, stall_test) == offsetof(BGlobal, wait_limit) + sizeof(unsigned),
                "wait_limit and stall_test are adjacent");
  SGB_CK(cudaMemcpyAsync(B->ws + B->o_g + offsetof(BGlobal, wait_limit), v, sizeof(v),
                         cudaMemcpyHostToDevice, s));
  SGB_CK(cudaStreamSynchronize(s));
  return SGH_OK;
}

int sgh_batch_volume_pass(sgh_batch* B, void* stream) {
  if (!B || !B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (B->precision == SGH_PRECISION_MIXED)
    launch_volume<float, true>(B, s, reinterpret_cast<float*>(B->ws + B->o_a), nullptr, nullptr);
  else
    launch_volume<double, true>(B, s, B->d(B->o_a), B->d(B->o_K), B->d(B->o_KK));
  SGB_CK(cudaGetLastError());
  return SGH_OK;
}

int sgh_batch_launch_counts(const sgh_batch* B, int32_t* pre, int32_t* per_iter, int32_t* post) {
  if (!B || !pre || !per_iter || !post) return bfail(SGH_ERR_INVALID, "null argument");
  if (!B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  *pre = B->n_pre;
  *per_iter = B->n_iter;
  *post = B->n_post;  // sgh_batch_step adds one run-setup kernel per call
  return SGH_OK;
}

}  // extern "C"
