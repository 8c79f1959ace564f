// sgh_batch.cu -- many instances of uneven size stepped together.
//
// Every stage of the time step runs as ONE launch over all slots of a batch.
// Work is decomposed per slot: element/column kernels give each slot
// ceil(S_i / 256) blocks, face transforms give each slot its 16 x 16 output
// tiles; a block finds its slot by binary search in a prefix table. Per-slot
// reductions (P_laser, Picard norms, surface max) are per-block partials that
// a single-block kernel sums slot by slot in a fixed order.
//
// The physics is the face-space Picard form (see sgh_b200.cu): every iterate
// of a slot is aK + KK Ct[p] sigma[y,x], so each step reads the modes twice
// (K a and the face sums; the commit) and the Picard loop runs on faces. The
// loop is a conditional graph node that repeats while any slot is still
// iterating; converged (or inactive) slots skip every kernel of the body, so
// a slot's result does not depend on what else is in the batch.
//
// Volume state (modes a, K, KK) is FP64 (plain) or FP32 (mixed: K/KK computed
// in FP64 and rounded once; all arithmetic on them in FP64 registers). Faces,
// face sums and norms are FP64 in both.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "sgh_b200.h"
#include "sgh_axis.cuh"
#include "sgh_device.cuh"
#include "sgh_umma.cuh"

namespace sgh {
namespace batch {

constexpr int BT = 256;   // threads of element / column / face kernels
constexpr int FT = 16;    // face transform tile edge
constexpr int CT = 1024;  // threads of the per-slot control kernels

struct BSlot {
  int nx, ny, nz, S;
  long long V;
  int max_iter, cell_integrated;
  long long vol;   // element offset of this slot in the volume arenas
  long long face;  // element offset in the face arenas
  int zoff;        // offset in the Ct table
  int mx, my;      // element offsets of the x / y DCT matrices (M, then M^T)
  int blk0, nblk;  // element / column blocks
  int tile0, ntile;  // face transform tiles
  int vblk0, nvblk;  // volume blocks (setup kernels)
  int utile0, nutile;  // tensor-core face tiles (mixed precision)
  long long xa, yb;    // byte offsets of the slot's x-pass A plane and y-pass B plane
  long long mpx, mpy;  // byte offsets of the forward x / y matrix planes (inverse at + mp_inv)
  long long mpx_inv, mpy_inv;
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
  int iter, done, status, pad;
  double I0, shift_x, shift_y, rel_err;
  sgh_step_out last;
};

struct BGlobal {
  int steps_left;
  int umma_err;     // nonzero once a tensor-core wait expired
  int picard_any;   // some slot is still iterating (read by the eager step)
  int pad;
};

// Device view of a bound batch (passed by value to every kernel).
struct BView {
  const BSlot* slot;
  BState* st;
  BGlobal* g;
  const int* blk_start;   // n + 1
  const int* tile_start;  // n + 1
  const int* vblk_start;  // n + 1
  const int* utile_start; // n + 1 (tensor-core face tiles)
  __nv_bfloat16* xa_hi;   // operand planes (mixed precision; null otherwise)
  __nv_bfloat16* xa_lo;
  __nv_bfloat16* yb_hi;
  __nv_bfloat16* yb_lo;
  const char* mp_hi;      // DCT matrix planes
  const char* mp_lo;
  const double* mats;
  const double* Ct;
  int n;
};

__device__ __forceinline__ int find_slot(const int* start, int n, int b) {
  int lo = 0, hi = n;  // largest s with start[s] <= b
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

// x-pass A-operand plane element (y, x) of slot sl (mixed precision only).
__device__ __forceinline__ void xa_put(const BView& v, const BSlot& sl, int y, int x, double val) {
  if (!v.xa_hi) return;
  const int nkc = (sl.nx + umma::KC - 1) / umma::KC;
  umma::plane_put(v.xa_hi + sl.xa / 2, v.xa_lo + sl.xa / 2, y, x, nkc, val);
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

// BF16 hi/lo planes of an N x N DCT matrix (inv: its transpose), rows = the
// output index, k = the contracted index.
__global__ void kb_matrix_planes(int N, const double* M, int inv, __nv_bfloat16* hi, __nv_bfloat16* lo) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * N) return;
  const int r = e / N, k = e - r * N;
  const double val = inv ? M[(size_t)k * N + r] : M[(size_t)r * N + k];
  umma::plane_put(hi, lo, r, k, (N + umma::KC - 1) / umma::KC, val);
}

// K, KK of every slot exactly as precompute_K_KK (physics/spectral_state.py:374-421),
// in FP64, stored as R; Ct tables.
template <class R>
__global__ void __launch_bounds__(BT) kb_tables(BView v, R* K, R* KK, double* Ct) {
  const int b = blockIdx.x;
  const int s = find_slot(v.vblk_start, v.n, b);
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
    K[sl.vol + i] = (R)k;
    KK[sl.vol + i] = (R)((i == 0) ? sl.dt / rho_cp : ((k - 1.0) / (-lam)) / rho_cp);
    if (i < sl.nz) {
      const double c = (i == 0) ? sqrt(1.0 / sl.Lz) : sqrt(2.0 / sl.Lz);
      Ct[sl.zoff + i] = (i & 1) ? -c : c;
    }
  }
}

// Face weights from the stored KK: W_tt = sum Ct^2 KK, Q_tt = sum (KK Ct)^2.
template <class R>
__global__ void __launch_bounds__(BT) kb_weights(BView v, const R* KK, double* Wtt, double* Qtt) {
  const int b = blockIdx.x;
  const int s = find_slot(v.blk_start, v.n, b);
  const BSlot& sl = v.slot[s];
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  if (i >= sl.S) return;
  double w = 0.0, q = 0.0;
  for (int p = 0; p < sl.nz; ++p) {
    const double kk = (double)KK[sl.vol + (long long)p * sl.S + i];
    const double ct = v.Ct[sl.zoff + p];
    w += ct * ct * kk;
    q += (kk * ct) * (kk * ct);
  }
  Wtt[sl.face + i] = w;
  Qtt[sl.face + i] = q;
}

// (Re)start one slot at the initial condition (solvers/spectral.py:176-180).
template <class R>
__global__ void __launch_bounds__(BT)
kb_slot_start(BView v, int s, R* a, double* q_evold, double* q_ev, double* sigma, const sgh_laser* table,
              int n_steps, sgh_step_out* outs) {
  const BSlot& sl = v.slot[s];
  const long long i = (long long)blockIdx.x * BT + threadIdx.x;
  if (i < sl.V) a[sl.vol + i] = (R)((i == 0) ? sl.T0 * sqrt(sl.Lx * sl.Ly * sl.Lz) : 0.0);
  if (i < sl.S) {
    q_evold[sl.face + i] = 0.0;
    q_ev[sl.face + i] = 0.0;
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
  }
}

__global__ void kb_slot_stop(BView v, int s) { v.st[s].active = 0; }

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
    st.shift_x = (L.vx * sl.dt) / sl.dx;
    st.shift_y = (L.vy * sl.dt) / sl.dy;
    st.iter = 0;
    st.status = SGH_STEP_CAPPED;
    st.rel_err = nan("");
    st.done = sl.max_iter > 0 ? 0 : 1;
    if (!st.done) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v.g->picard_any = any;
    if (in_graph) cudaGraphSetConditional(h_picard, any ? 1u : 0u);
  }
}

// q_las, P_laser partials and q_net = q_las - shift(q_evap_old) per slot
// (solvers/spectral.py:273-306).
__global__ void __launch_bounds__(BT)
kb_face_begin(BView v, double* q_las, double* q_net, const double* q_evold, double* part_las) {
  __shared__ double sh[2 * (BT / 32)];
  const int b = blockIdx.x;
  const int s = find_slot(v.blk_start, v.n, b);
  const BSlot& sl = v.slot[s];
  const BState& st = v.st[s];
  if (!st.active) return;
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  double sum = 0.0, dummy = 0.0;
  if (i < sl.S) {
    const int nx = sl.nx, ny = sl.ny;
    const int y = i / nx, x = i - y * nx;
    const double xc = ((double)x + 0.5) * sl.dx, yc = ((double)y + 0.5) * sl.dy;
    const double q = laser_flux(sl, st.I0, st.laser.x, st.laser.y, xc, yc);
    const double* f = q_evold + sl.face;
    q_las[sl.face + i] = q;
    sum = q;
    const ShiftTap ty = shift_tap(y, ny, st.shift_y);
    const ShiftTap tx = shift_tap(x, nx, st.shift_x);
    double val = ty.w0 * (tx.w0 * f[ty.i0 * nx + tx.i0] + tx.w1 * f[ty.i0 * nx + tx.i1]) +
                 ty.w1 * (tx.w0 * f[ty.i1 * nx + tx.i0] + tx.w1 * f[ty.i1 * nx + tx.i1]);
    if (!(ty.in && tx.in)) val = 0.0;
    q_net[sl.face + i] = q - val;
    xa_put(v, sl, y, x, q - val);
  }
  block_sum2<BT>(sum, dummy, sh);
  if (threadIdx.x == 0) part_las[b] = sum;
}

// Face sums of the propagated modes: Zt = sum Ct K a, Yt = sum (K a) KK Ct and
// partials of sum (K a)^2.
template <class R>
__global__ void __launch_bounds__(BT)
kb_pass1(BView v, const R* a, const R* K, const R* KK, double* Zt, double* Yt, double* part_n1) {
  __shared__ double sh[2 * (BT / 32)];
  const int b = blockIdx.x;
  const int s = find_slot(v.blk_start, v.n, b);
  const BSlot& sl = v.slot[s];
  if (!v.st[s].active) return;
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  double n1 = 0.0, dummy = 0.0;
  if (i < sl.S) {
    double zt = 0.0, yt = 0.0;
    const double* ct = v.Ct + sl.zoff;
    for (int p = 0; p < sl.nz; ++p) {
      const long long j = sl.vol + (long long)p * sl.S + i;
      const double ak = (double)a[j] * (double)K[j];
      const double kk = (double)KK[j];
      zt = fma(ct[p], ak, zt);
      yt = fma(ak * kk, ct[p], yt);
      n1 = fma(ak, ak, n1);
    }
    Zt[sl.face + i] = zt;
    Yt[sl.face + i] = yt;
  }
  block_sum2<BT>(n1, dummy, sh);
  if (threadIdx.x == 0) part_n1[b] = n1;
}

// A = Zt + W_tt sigma (top-surface input of the current iterate).
__global__ void __launch_bounds__(BT)
kb_assemble(BView v, const double* Zt, const double* Wtt, const double* sigma, double* A) {
  const int b = blockIdx.x;
  const int s = find_slot(v.blk_start, v.n, b);
  const BSlot& sl = v.slot[s];
  if (!v.st[s].active) return;
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  if (i < sl.S) {
    const double a = Zt[sl.face + i] + Wtt[sl.face + i] * sigma[sl.face + i];
    A[sl.face + i] = a;
    xa_put(v, sl, i / sl.nx, i % sl.nx, a);
  }
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
  const int s = find_slot(v.tile_start, v.n, b);
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

// ---- batched face transform on the tensor cores (mixed precision) ---------
// Same contraction as kb_face_axis, as 128 x UNT tiles of split-BF16 products
// accumulated in FP32 in tensor memory (sgh_umma.cuh); slot tiles:
// ceil(ny / 128) * ceil(nx / UNT) in both directions.
constexpr int UNT = 128;
inline __host__ __device__ int face_utiles(int nx, int ny) {
  return ((ny + umma::TM - 1) / umma::TM) * ((nx + UNT - 1) / UNT);
}

struct ULoadX {  // DIR 0, A(m = y, k = n) = in[y][n]
  const double* p;
  int nx;
  __device__ __forceinline__ double operator()(int m, int k) const { return p[(size_t)m * nx + k]; }
};
struct ULoadM {  // matrix rows: M(r, k) = M[r * N + k]
  const double* p;
  int N;
  __device__ __forceinline__ double operator()(int r, int k) const { return p[(size_t)r * N + k]; }
};
struct ULoadT {  // DIR 1, B(n = x, k = n') = in[n'][x]
  const double* p;
  int nx;
  __device__ __forceinline__ double operator()(int r, int k) const { return p[(size_t)k * nx + r]; }
};

template <class Epi>
struct UEpi {  // (m, n, v) -> batched epilogue on face index m * nx + n
  const BSlot* sl;
  BState* st;
  Epi e;
  Red* r;
  __device__ __forceinline__ void operator()(int m, int n, double v) const {
    e(*sl, *st, sl->face + (long long)m * sl->nx + n, v, *r);
  }
};

template <int DIR, bool INV, bool SKIP_DONE, class Epi>
__global__ void __launch_bounds__(umma::THREADS)
kb_face_umma(BView v, const double* in, Epi epi, double* part_tile) {
  extern __shared__ __align__(128) char usmem[];
  __shared__ double red[umma::THREADS / 32];
  const int b = blockIdx.x;
  const int s = find_slot(v.utile_start, v.n, b);
  const BSlot& sl = v.slot[s];
  BState& st = v.st[s];
  if (!st.active || (SKIP_DONE && st.done)) return;
  const int t = b - sl.utile0;
  const int nx = sl.nx, ny = sl.ny;
  const int nct = (nx + UNT - 1) / UNT;
  const int n0 = (t % nct) * UNT, m0 = (t / nct) * umma::TM;
  const int N = DIR == 0 ? nx : ny;
  const double* M = v.mats + (DIR == 0 ? sl.mx : sl.my) + (INV ? (size_t)N * N : 0);
  const double* X = in + sl.face;
  Red r;
  UEpi<Epi> ue{&sl, &st, epi, &r};
  if (DIR == 0)
    umma::tile_bf16x3<UNT>(ny, nx, nx, m0, n0, ULoadX{X, nx}, ULoadM{M, nx}, ue, usmem, &v.g->umma_err);
  else
    umma::tile_bf16x3<UNT>(ny, nx, ny, m0, n0, ULoadM{M, ny}, ULoadT{X, nx}, ue, usmem, &v.g->umma_err);
  if (Epi::kMax) {
    double m = r.mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = red[0];
      for (int w = 1; w < umma::THREADS / 32; ++w) mm = fmax(mm, red[w]);
      part_tile[b] = mm;
    }
  }
}

// ---- batched face transform fed from operand planes (mixed precision) ---
// DIR 0 (x-pass): A = the slot's x-pass plane (rows y, k = x), B = the x
// matrix plane (rows k, k = n); DIR 1 (y-pass): A = the y matrix plane, B =
// the slot's y-pass plane (rows x, k = y). epi(sl, st, m, n, value, r) gets
// every in-range element, (m, n) = (y, k) for DIR 0 and (k, x) for DIR 1.
template <int DIR, bool INV, bool SKIP_DONE, class Epi>
__global__ void __launch_bounds__(umma::THREADS) kb_face_tc(BView v, Epi epi, double* part_tile) {
  extern __shared__ __align__(128) char usmem[];
  __shared__ double red[umma::THREADS / 32];
  const int b = blockIdx.x;
  const int s = find_slot(v.utile_start, v.n, b);
  const BSlot& sl = v.slot[s];
  BState& st = v.st[s];
  if (!st.active || (SKIP_DONE && st.done)) return;
  const int t = b - sl.utile0;
  const int nx = sl.nx, ny = sl.ny;
  const int nct = (nx + UNT - 1) / UNT;
  const int rt = t / nct, ct = t % nct;
  const int nkc = ((DIR == 0 ? nx : ny) + umma::KC - 1) / umma::KC;
  const size_t cb = (size_t)umma::CHUNK_BYTES;
  const char *ah, *al, *bh, *bl;
  if (DIR == 0) {
    ah = reinterpret_cast<const char*>(v.xa_hi) + sl.xa + rt * nkc * cb;
    al = reinterpret_cast<const char*>(v.xa_lo) + sl.xa + rt * nkc * cb;
    const long long mp = INV ? sl.mpx_inv : sl.mpx;
    bh = v.mp_hi + mp + ct * nkc * cb;
    bl = v.mp_lo + mp + ct * nkc * cb;
  } else {
    const long long mp = INV ? sl.mpy_inv : sl.mpy;
    ah = v.mp_hi + mp + rt * nkc * cb;
    al = v.mp_lo + mp + rt * nkc * cb;
    bh = reinterpret_cast<const char*>(v.yb_hi) + sl.yb + ct * nkc * cb;
    bl = reinterpret_cast<const char*>(v.yb_lo) + sl.yb + ct * nkc * cb;
  }
  Red r;
  const int m0 = rt * umma::TM, n0 = ct * UNT;
  const int Mrows = ny;  // both directions: rows y (DIR 0) or k over ny (DIR 1)
  auto tepi = [&](int ml, int nl, double val) {
    const int m = m0 + ml, n = n0 + nl;
    if (m < Mrows && n < nx) epi(v, sl, st, m, n, val, r);
  };
  umma::tile_planes(ah, al, bh, bl, nkc, tepi, usmem, &v.g->umma_err);
  if (Epi::kMax) {
    double m = r.mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = red[0];
      for (int w = 1; w < umma::THREADS / 32; ++w) mm = fmax(mm, red[w]);
      part_tile[b] = mm;
    }
  }
}

struct TE_ToYB {  // x-pass result (y, k) -> y-pass B plane element (row k, k-index y)
  static constexpr int kMax = 0;
  __device__ __forceinline__ void operator()(const BView& v, const BSlot& sl, const BState&, int y, int k,
                                             double val, Red&) const {
    const int nkc = (sl.ny + umma::KC - 1) / umma::KC;
    umma::plane_put(v.yb_hi + sl.yb / 2, v.yb_lo + sl.yb / 2, k, y, nkc, val);
  }
};
struct TE_Store {  // y-pass result -> FP64 face array (times dct_scale if scaled)
  static constexpr int kMax = 0;
  double* out;
  int scaled;
  __device__ __forceinline__ void operator()(const BView&, const BSlot& sl, const BState&, int k, int x,
                                             double val, Red&) const {
    out[sl.face + (long long)k * sl.nx + x] = scaled ? val * sl.dct_scale : val;
  }
};
struct TE_TopFlux {  // T_s -> evaporation -> q_net into the x-pass A plane (solvers/spectral.py:388-404)
  static constexpr int kMax = 0;
  const double* q_las;
  double* q_ev;
  double* q_net;
  __device__ __forceinline__ void operator()(const BView& v, const BSlot& sl, const BState&, int y, int x,
                                             double val, Red&) const {
    const long long i = sl.face + (long long)y * sl.nx + x;
    const double Ts = sl.recon_scale * val;
    const double qe = evaporation(sl, Ts);
    q_ev[i] = qe;
    const double qn = q_las[i] - qe;
    q_net[i] = qn;
    xa_put(v, sl, y, x, qn);
  }
};
struct TE_CommitSurface {  // T_temp, its max, q_evap_old <- q_evap
  static constexpr int kMax = 1;
  double* T_surf;
  const double* q_ev;
  double* q_evold;
  __device__ __forceinline__ void operator()(const BView&, const BSlot& sl, const BState&, int y, int x,
                                             double val, Red& r) const {
    const long long i = sl.face + (long long)y * sl.nx + x;
    const double T = sl.recon_scale * val;
    T_surf[i] = T;
    q_evold[i] = q_ev[i];
    r.mx = fmax(r.mx, T);
  }
};

struct EB_Store {  // out = v * (scaled ? dct_scale : 1)
  static constexpr int kMax = 0;
  double* out;
  int scaled;
  __device__ __forceinline__ void operator()(const BSlot& sl, const BState&, long long i, double v, Red&) const {
    out[i] = scaled ? v * sl.dct_scale : v;
  }
};

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

struct EB_CommitSurface {  // T_temp, its max, q_evap_old <- q_evap (solvers/spectral.py:502-512)
  static constexpr int kMax = 1;
  double* T_surf;
  const double* q_ev;
  double* q_evold;
  __device__ __forceinline__ void operator()(const BSlot& sl, const BState&, long long i, double v, Red& r) const {
    const double T = sl.recon_scale * v;
    T_surf[i] = T;
    q_evold[i] = q_ev[i];
    r.mx = fmax(r.mx, T);
  }
};

// Face-state update of one Picard iteration (see k_fs_relax in sgh_b200.cu):
// residual and iterate norms from the constant weights, relaxation of sigma.
__global__ void __launch_bounds__(BT)
kb_relax(BView v, const double* Zt, const double* Yt, const double* Wtt, const double* Qtt,
         const double* S_top, double* sigma, double* A, double* part) {
  __shared__ double sh[2 * (BT / 32)];
  const int b = blockIdx.x;
  const int s = find_slot(v.blk_start, v.n, b);
  const BSlot& sl = v.slot[s];
  const BState& st = v.st[s];
  if (!st.active || st.done) return;
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  double r2 = 0.0, o2 = 0.0;
  if (i < sl.S) {
    const long long j = sl.face + i;
    const double sg = sigma[j], q = Qtt[j];
    const double d = S_top[j] - sg;
    r2 = d * d * q;
    o2 = 2.0 * sg * Yt[j] + sg * sg * q;
    const double ns = d * sl.omega + sg;
    sigma[j] = ns;
    const double a = Zt[j] + Wtt[j] * ns;
    A[j] = a;
    xa_put(v, sl, i / sl.nx, i % sl.nx, a);
  }
  block_sum2<BT>(r2, o2, sh);
  if (threadIdx.x == 0) {
    part[2 * b] = r2;
    part[2 * b + 1] = o2;
  }
}

// Per-slot convergence test (solvers/spectral.py:464-499); the loop goes on
// while any slot is still iterating.
__global__ void __launch_bounds__(CT)
kb_converge(BView v, const double* part, const double* part_n1, cudaGraphConditionalHandle h_picard,
            int in_graph) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < v.n; s += CT) {
    BState& st = v.st[s];
    if (!st.active || st.done) continue;
    const BSlot& sl = v.slot[s];
    double r2 = 0.0, o2 = 0.0;
    for (int b = sl.blk0; b < sl.blk0 + sl.nblk; ++b) {
      r2 += part[2 * b];
      o2 += part[2 * b + 1] + part_n1[b];
    }
    const double n = sl.n_elements;
    const double rel = sqrt(r2 / n) / fmax(sqrt(o2 / n), 1e-9);
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
    if (!st.done) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v.g->picard_any = any;
    if (in_graph) cudaGraphSetConditional(h_picard, any ? 1u : 0u);
  }
}

// a = K a + KK Ct sigma (commit of the modes).
template <class R>
__global__ void __launch_bounds__(BT)
kb_commit_modes(BView v, R* a, const R* K, const R* KK, const double* sigma) {
  const int b = blockIdx.x;
  const int s = find_slot(v.blk_start, v.n, b);
  const BSlot& sl = v.slot[s];
  if (!v.st[s].active) return;
  const int i = (b - sl.blk0) * BT + threadIdx.x;
  if (i >= sl.S) return;
  const double sg = sigma[sl.face + i];
  const double* ct = v.Ct + sl.zoff;
  for (int p = 0; p < sl.nz; ++p) {
    const long long j = sl.vol + (long long)p * sl.S + i;
    a[j] = (R)((double)a[j] * (double)K[j] + (double)KK[j] * (ct[p] * sg));
  }
}

// Metrics of every active slot (solvers/spectral.py:536-542); advances the
// step counters and decides whether the step loop continues.
__global__ void __launch_bounds__(CT)
kb_commit(BView v, const double* part_las, const double* part_tile, int umma_tiles,
          cudaGraphConditionalHandle h_steps, int in_graph) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < v.n; s += CT) {
    BState& st = v.st[s];
    if (!st.active) continue;
    const BSlot& sl = v.slot[s];
    double p = 0.0, m = -INFINITY;
    for (int b = sl.blk0; b < sl.blk0 + sl.nblk; ++b) p += part_las[b];
    const int t0 = umma_tiles ? sl.utile0 : sl.tile0, nt = umma_tiles ? sl.nutile : sl.ntile;
    for (int b = t0; b < t0 + nt; ++b) m = fmax(m, part_tile[b]);
    sgh_step_out o;
    o.T_surface_max = m;
    o.P_laser = p * sl.dx * sl.dy;
    o.picard_rel_err = st.rel_err;
    o.n_iter = st.iter;
    o.converged = st.status == SGH_STEP_CONVERGED ? 1 : 0;
    o.status = st.status;
    o.pad = 0;
    st.last = o;
    if (st.outs) st.outs[st.step] = o;
    st.iters += st.iter;
    st.step += 1;
    if (st.step >= st.n_steps) st.active = 0;
    if (st.active) any = 1;
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
  std::vector<int> blk_start, tile_start, vblk_start, utile_start;
  std::vector<std::pair<int, long long>> mat_list;  // (N, element offset)
  long long tot_vol = 0, tot_face = 0;
  int tot_blk = 0, tot_tile = 0, tot_vblk = 0, tot_z = 0, tot_utile = 0;
  long long mat_elems = 0;
  // workspace offsets (bytes)
  size_t o_slot, o_state, o_g, o_blk, o_tile, o_vblk, o_utile, o_mats, o_ct;
  size_t o_a, o_K, o_KK;
  size_t o_qlas, o_qnet, o_qev, o_qevold, o_Stop, o_f1, o_sigma, o_A, o_Tsurf, o_Zt, o_Yt, o_Wtt, o_Qtt;
  size_t o_plas, o_pn1, o_prelax, o_ptile;
  size_t o_xah = 0, o_xal = 0, o_ybh = 0, o_ybl = 0, o_mph = 0, o_mpl = 0;  // operand planes (mixed)
  size_t xa_bytes = 0, yb_bytes = 0, mp_bytes = 0;
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
  BView view() const {
    BView v;
    v.slot = reinterpret_cast<const BSlot*>(ws + o_slot);
    v.st = reinterpret_cast<BState*>(ws + o_state);
    v.g = reinterpret_cast<BGlobal*>(ws + o_g);
    v.blk_start = reinterpret_cast<const int*>(ws + o_blk);
    v.tile_start = reinterpret_cast<const int*>(ws + o_tile);
    v.vblk_start = reinterpret_cast<const int*>(ws + o_vblk);
    v.utile_start = reinterpret_cast<const int*>(ws + o_utile);
    const bool mixed = precision == SGH_PRECISION_MIXED;
    v.xa_hi = mixed ? reinterpret_cast<__nv_bfloat16*>(ws + o_xah) : nullptr;
    v.xa_lo = mixed ? reinterpret_cast<__nv_bfloat16*>(ws + o_xal) : nullptr;
    v.yb_hi = mixed ? reinterpret_cast<__nv_bfloat16*>(ws + o_ybh) : nullptr;
    v.yb_lo = mixed ? reinterpret_cast<__nv_bfloat16*>(ws + o_ybl) : nullptr;
    v.mp_hi = mixed ? ws + o_mph : nullptr;
    v.mp_lo = mixed ? ws + o_mpl : nullptr;
    v.mats = d(o_mats);
    v.Ct = d(o_ct);
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

// One face pass over all slots: the FP64 register-tiled contraction on the
// FP64 input (plain), or tensor-core split-BF16 tiles fed by bulk copies
// from the operand planes (mixed).
template <int DIR, bool INV, bool SKIP, class EpiF, class EpiT>
void face_pass(sgh_batch* B, cudaStream_t s, const double* in, const EpiF& ef, const EpiT& et, double* part) {
  const BView v = B->view();
  if (B->precision == SGH_PRECISION_MIXED) {
    const int smem = umma::planes_smem_bytes();
    (void)cudaFuncSetAttribute(kb_face_tc<DIR, INV, SKIP, EpiT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    kb_face_tc<DIR, INV, SKIP, EpiT><<<B->tot_utile, umma::THREADS, smem, s>>>(v, et, part);
  } else {
    kb_face_axis<DIR, INV, SKIP, EpiF><<<B->tot_tile, AX_THREADS, 0, s>>>(v, in, ef, part);
  }
  ++g_blaunch;
}

template <class R>
void enqueue_pre(sgh_batch* B, cudaStream_t s, cudaGraphConditionalHandle h, int in_graph) {
  const BView v = B->view();
  R* a = reinterpret_cast<R*>(B->ws + B->o_a);
  R* K = reinterpret_cast<R*>(B->ws + B->o_K);
  R* KK = reinterpret_cast<R*>(B->ws + B->o_KK);
  kb_begin<<<1, CT, 0, s>>>(v, h, in_graph);
  kb_face_begin<<<B->tot_blk, BT, 0, s>>>(v, B->d(B->o_qlas), B->d(B->o_qnet), B->d(B->o_qevold), B->d(B->o_plas));
  kb_pass1<R><<<B->tot_blk, BT, 0, s>>>(v, a, K, KK, B->d(B->o_Zt), B->d(B->o_Yt), B->d(B->o_pn1));
  g_blaunch += 3;
  // initial guess: sigma = dct_scale * DCT2(q_las - shift(q_evap_old))
  face_pass<0, false, false>(B, s, B->d(B->o_qnet), EB_Store{B->d(B->o_f1), 0}, TE_ToYB{}, nullptr);
  face_pass<1, false, false>(B, s, B->d(B->o_f1), EB_Store{B->d(B->o_sigma), 1}, TE_Store{B->d(B->o_sigma), 1},
                             nullptr);
  kb_assemble<<<B->tot_blk, BT, 0, s>>>(v, B->d(B->o_Zt), B->d(B->o_Wtt), B->d(B->o_sigma), B->d(B->o_A));
  g_blaunch += 1;
}

void enqueue_picard(sgh_batch* B, cudaStream_t s, cudaGraphConditionalHandle h, int in_graph) {
  const BView v = B->view();
  face_pass<0, true, true>(B, s, B->d(B->o_A), EB_Store{B->d(B->o_f1), 0}, TE_ToYB{}, nullptr);
  face_pass<1, true, true>(B, s, B->d(B->o_f1), EB_TopFlux{B->d(B->o_qlas), B->d(B->o_qev), B->d(B->o_qnet)},
                           TE_TopFlux{B->d(B->o_qlas), B->d(B->o_qev), B->d(B->o_qnet)}, nullptr);
  face_pass<0, false, true>(B, s, B->d(B->o_qnet), EB_Store{B->d(B->o_f1), 0}, TE_ToYB{}, nullptr);
  face_pass<1, false, true>(B, s, B->d(B->o_f1), EB_Store{B->d(B->o_Stop), 1}, TE_Store{B->d(B->o_Stop), 1},
                            nullptr);
  kb_relax<<<B->tot_blk, BT, 0, s>>>(v, B->d(B->o_Zt), B->d(B->o_Yt), B->d(B->o_Wtt), B->d(B->o_Qtt),
                                     B->d(B->o_Stop), B->d(B->o_sigma), B->d(B->o_A), B->d(B->o_prelax));
  kb_converge<<<1, CT, 0, s>>>(v, B->d(B->o_prelax), B->d(B->o_pn1), h, in_graph);
  g_blaunch += 2;
}

template <class R>
void enqueue_post(sgh_batch* B, cudaStream_t s, cudaGraphConditionalHandle h, int in_graph) {
  const BView v = B->view();
  R* a = reinterpret_cast<R*>(B->ws + B->o_a);
  R* K = reinterpret_cast<R*>(B->ws + B->o_K);
  R* KK = reinterpret_cast<R*>(B->ws + B->o_KK);
  face_pass<0, true, false>(B, s, B->d(B->o_A), EB_Store{B->d(B->o_f1), 0}, TE_ToYB{}, nullptr);
  face_pass<1, true, false>(B, s, B->d(B->o_f1),
                            EB_CommitSurface{B->d(B->o_Tsurf), B->d(B->o_qev), B->d(B->o_qevold)},
                            TE_CommitSurface{B->d(B->o_Tsurf), B->d(B->o_qev), B->d(B->o_qevold)},
                            B->d(B->o_ptile));
  kb_commit_modes<R><<<B->tot_blk, BT, 0, s>>>(v, a, K, KK, B->d(B->o_sigma));
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
      mplane[kv.first] = po;
      B->mplane_list.push_back({kv.first, po});
      po += 2LL * (long long)umma::plane_bytes(kv.first, kv.first);
    }
    B->mp_bytes = (size_t)po;
  }
  B->blk_start.assign(n + 1, 0);
  B->tile_start.assign(n + 1, 0);
  B->vblk_start.assign(n + 1, 0);
  B->utile_start.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    const sgh_config& c = cfgs[i];
    BSlot sl;
    std::memset(&sl, 0, sizeof(sl));
    sl.nx = c.nx; sl.ny = c.ny; sl.nz = c.nz;
    sl.S = c.nx * c.ny;
    sl.V = (long long)sl.S * c.nz;
    sl.max_iter = c.max_iter;
    sl.cell_integrated = c.cell_integrated;
    sl.vol = B->tot_vol;
    sl.face = B->tot_face;
    sl.zoff = B->tot_z;
    sl.mx = (int)mats[c.nx];
    sl.my = (int)mats[c.ny];
    sl.blk0 = B->tot_blk;
    sl.nblk = cdivl(sl.S, BT);
    sl.tile0 = B->tot_tile;
    sl.ntile = face_tiles(c.nx, c.ny);
    sl.vblk0 = B->tot_vblk;
    sl.nvblk = cdivl(sl.V, BT);
    sl.utile0 = B->tot_utile;
    sl.nutile = face_utiles(c.nx, c.ny);
    if (precision == SGH_PRECISION_MIXED) {
      sl.xa = (long long)B->xa_bytes;
      sl.yb = (long long)B->yb_bytes;
      B->xa_bytes += umma::plane_bytes(c.ny, c.nx);
      B->yb_bytes += umma::plane_bytes(c.nx, c.ny);
      sl.mpx = mplane[c.nx];
      sl.mpx_inv = sl.mpx + (long long)umma::plane_bytes(c.nx, c.nx);
      sl.mpy = mplane[c.ny];
      sl.mpy_inv = sl.mpy + (long long)umma::plane_bytes(c.ny, c.ny);
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
    B->tot_vol += sl.V;
    B->tot_face += sl.S;
    B->tot_z += c.nz;
    B->tot_blk += sl.nblk;
    B->tot_tile += sl.ntile;
    B->tot_vblk += sl.nvblk;
    B->tot_utile += sl.nutile;
    B->blk_start[i + 1] = B->tot_blk;
    B->tile_start[i + 1] = B->tot_tile;
    B->vblk_start[i + 1] = B->tot_vblk;
    B->utile_start[i + 1] = B->tot_utile;
  }
  LayoutB L;
  const size_t F8 = sizeof(double) * (size_t)B->tot_face;
  const size_t VE = B->elem() * (size_t)B->tot_vol;
  B->o_slot = L.take(sizeof(BSlot) * n);
  B->o_state = L.take(sizeof(BState) * n);
  B->o_g = L.take(sizeof(BGlobal));
  B->o_blk = L.take(sizeof(int) * (n + 1));
  B->o_tile = L.take(sizeof(int) * (n + 1));
  B->o_vblk = L.take(sizeof(int) * (n + 1));
  B->o_utile = L.take(sizeof(int) * (n + 1));
  B->o_mats = L.take(sizeof(double) * (size_t)B->mat_elems);
  B->o_ct = L.take(sizeof(double) * (size_t)B->tot_z);
  B->o_a = L.take(VE);
  B->o_K = L.take(VE);
  B->o_KK = L.take(VE);
  B->o_qlas = L.take(F8);
  B->o_qnet = L.take(F8);
  B->o_qev = L.take(F8);
  B->o_qevold = L.take(F8);
  B->o_Stop = L.take(F8);
  B->o_f1 = L.take(F8);
  B->o_sigma = L.take(F8);
  B->o_A = L.take(F8);
  B->o_Tsurf = L.take(F8);
  B->o_Zt = L.take(F8);
  B->o_Yt = L.take(F8);
  B->o_Wtt = L.take(F8);
  B->o_Qtt = L.take(F8);
  B->o_plas = L.take(sizeof(double) * B->tot_blk);
  B->o_pn1 = L.take(sizeof(double) * B->tot_blk);
  B->o_prelax = L.take(sizeof(double) * 2 * B->tot_blk);
  B->o_ptile = L.take(sizeof(double) * std::max(B->tot_tile, B->tot_utile));
  if (precision == SGH_PRECISION_MIXED) {
    B->o_xah = L.take(B->xa_bytes);
    B->o_xal = L.take(B->xa_bytes);
    B->o_ybh = L.take(B->yb_bytes);
    B->o_ybl = L.take(B->yb_bytes);
    B->o_mph = L.take(B->mp_bytes);
    B->o_mpl = L.take(B->mp_bytes);
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
  SGB_CK(cudaMemcpyAsync(B->ws + B->o_blk, B->blk_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  SGB_CK(cudaMemcpyAsync(B->ws + B->o_tile, B->tile_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  SGB_CK(cudaMemcpyAsync(B->ws + B->o_vblk, B->vblk_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  SGB_CK(cudaMemcpyAsync(B->ws + B->o_utile, B->utile_start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  SGB_CK(cudaMemsetAsync(B->ws + B->o_qevold, 0, sizeof(double) * B->tot_face, s));
  SGB_CK(cudaMemsetAsync(B->ws + B->o_qev, 0, sizeof(double) * B->tot_face, s));
  for (auto& m : B->mat_list)
    kb_dct_matrix<<<cdivl((long long)m.first * m.first, BT), BT, 0, s>>>(m.first, B->d(B->o_mats) + m.second);
  const BView v = B->view();
  if (B->precision == SGH_PRECISION_MIXED) {
    SGB_CK(cudaMemsetAsync(B->ws + B->o_xah, 0, B->xa_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_xal, 0, B->xa_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_ybh, 0, B->yb_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_ybl, 0, B->yb_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_mph, 0, B->mp_bytes, s));
    SGB_CK(cudaMemsetAsync(B->ws + B->o_mpl, 0, B->mp_bytes, s));
    for (size_t j = 0; j < B->mplane_list.size(); ++j) {
      const int N = B->mplane_list[j].first;
      const long long po = B->mplane_list[j].second;
      long long moff = -1;
      for (auto& m : B->mat_list)
        if (m.first == N) moff = m.second;
      const size_t pb = umma::plane_bytes(N, N);
      for (int inv = 0; inv < 2; ++inv)
        kb_matrix_planes<<<cdivl((long long)N * N, BT), BT, 0, s>>>(
            N, B->d(B->o_mats) + moff, inv, reinterpret_cast<__nv_bfloat16*>(B->ws + B->o_mph + po + inv * pb),
            reinterpret_cast<__nv_bfloat16*>(B->ws + B->o_mpl + po + inv * pb));
    }
    float* K = reinterpret_cast<float*>(B->ws + B->o_K);
    float* KK = reinterpret_cast<float*>(B->ws + B->o_KK);
    kb_tables<float><<<B->tot_vblk, BT, 0, s>>>(v, K, KK, B->d(B->o_ct));
    kb_weights<float><<<B->tot_blk, BT, 0, s>>>(v, KK, B->d(B->o_Wtt), B->d(B->o_Qtt));
  } else {
    double* K = B->d(B->o_K);
    double* KK = B->d(B->o_KK);
    kb_tables<double><<<B->tot_vblk, BT, 0, s>>>(v, K, KK, B->d(B->o_ct));
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
                                          B->d(B->o_qevold), B->d(B->o_qev), B->d(B->o_sigma), lasers_dev,
                                          n_steps, outs_dev);
  else
    kb_slot_start<double><<<g, BT, 0, s>>>(B->view(), slot, B->d(B->o_a), B->d(B->o_qevold), B->d(B->o_qev),
                                           B->d(B->o_sigma), lasers_dev, n_steps, outs_dev);
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
    case SGH_BUF_K: off = B->o_K + e * sl.vol; nb = e * sl.V; break;
    case SGH_BUF_KK: off = B->o_KK + e * sl.vol; nb = e * sl.V; break;
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

int sgh_batch_launch_counts(const sgh_batch* B, int32_t* pre, int32_t* per_iter, int32_t* post) {
  if (!B || !pre || !per_iter || !post) return bfail(SGH_ERR_INVALID, "null argument");
  if (!B->bound) return bfail(SGH_ERR_STATE, "batch is not bound");
  *pre = B->n_pre;
  *per_iter = B->n_iter;
  *post = B->n_post;  // sgh_batch_step adds one run-setup kernel per call
  return SGH_OK;
}

}  // extern "C"
