// sgh_device.cuh -- device-side parameter block and pointwise physics of the
// time step. Every formula cites the reference routine it restates; all
// arithmetic is FP64 and follows the reference's operation order.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "sgh_b200.h"

namespace sgh {

// Program slots inside DevParams::prog.
enum { P_K_SOLID = 0, P_K_LIQUID, P_RHO_SOLID, P_RHO_LIQUID, P_C_SOLID, P_C_LIQUID, P_COUNT };

// Per-instance constants, built on the host from sgh_config and copied into
// the workspace once at bind time. Kernels read it through a const pointer.
struct DevParams {
  int nx, ny, nz, S, V;
  int grid_latent, prop_corr, latent_model, k_constant;
  int has_top_conv, has_bottom_conv, cell_integrated, max_iter;
  int degenerate_band;
  // box mode (FineMeshState, physics/spectral_state.py:166-239): box extents
  // xb, yb, zb (nx_box, ny_box, nz_box), fine-grid totals fx, fy, fz
  // (n_fine_totals), Nb = zb yb xb
  int box, xb, yb, zb, fx, fy, fz, Nb;
  int round32;  // mixed-precision plan: modal iterates rounded to FP32 at every write
  double Lx, Ly, Lz, dx, dy, dz, inv_dx, inv_dy, inv_dz, dt, inv_dt;
  double dct_scale, recon_scale, sqrt_dV, n_elements;
  double kbar, abar, T0, h_top, h_bottom;
  double evap_f1, evap_f2, T_boil, T_liquidus, T_solidus;
  double band_inv;          // 1/(T_l - T_s) (multiplication form of the kernels)
  double latent_factor;     // -rho L / dt (constant-property latent source)
  double L_f;
  double r_x, r_y, absorptivity, order, area_factor;
  double omega, tol;
  double dxf, dyf, dzf, dV_fine;  // fine spacings and cell volume (box mode)
  int affine[P_COUNT];       // program reduces to aff_a + aff_b * T (host analysis)
  double aff_a[P_COUNT], aff_b[P_COUNT];
  sgh_program prog[P_COUNT];
};

// Per-step control block (device resident; written by the step kernels).
struct Ctrl {
  sgh_laser laser;          // current laser state
  const sgh_laser* table;   // laser table (sgh_run) or null (sgh_step)
  sgh_step_out* out_table;  // metrics table (sgh_run) or null
  int n_target, step;       // steps requested / done in this launch
  int iter, stop;           // Picard iteration counter / loop-exit flag
  int have_qprev, status;
  double I0, shift_x, shift_y;  // peak intensity and warm-start shift (pixels)
  double rel_err;
  sgh_step_out out;         // metrics of the last step
  // box mode: history present (FineMeshState.T_prev is not None), window
  // start indices, history shift in fine pixels, and the magnitude maxima of
  // the committed latent source (peak, floor, x edges, y edges) as the bit
  // patterns of non-negative doubles (ordered like the values)
  int have_tprev, box_i0x, box_i0y, pad_c;
  double box_sx, box_sy;
  unsigned long long box_max[4];
  // Picard history of the current step: (rms of the residual, relative
  // residual) per iteration, the first hist_cap iterations
  double* hist;
  int hist_cap;
  int umma_err;  // a split-BF16 tensor-core wait ran out (mixed-precision plans)
};

// ---------------------------------------------------------------------------
// property programs (core/property_expr.py grammar; postfix, FP64)
// ---------------------------------------------------------------------------
// Kept out of line: inlined into every epilogue, the interpreter's switch
// (every math function of the grammar) evicts the hot loop from the
// instruction cache, although affine programs never reach it.
static __device__ __noinline__ double eval_program(const sgh_program& p, double T) {
  double st[SGH_MAX_STACK];
  int sp = 0;
  const int n = p.n_ops;
  for (int i = 0; i < n;) {
    const int op = p.ops[i++];
    switch (op) {
      case SGH_OP_CONST: st[sp++] = p.consts[p.ops[i++]]; break;
      case SGH_OP_T: st[sp++] = T; break;
      case SGH_OP_ADD: --sp; st[sp - 1] = st[sp - 1] + st[sp]; break;
      case SGH_OP_SUB: --sp; st[sp - 1] = st[sp - 1] - st[sp]; break;
      case SGH_OP_MUL: --sp; st[sp - 1] = st[sp - 1] * st[sp]; break;
      case SGH_OP_DIV: --sp; st[sp - 1] = st[sp - 1] / st[sp]; break;
      case SGH_OP_POW: --sp; st[sp - 1] = pow(st[sp - 1], st[sp]); break;
      case SGH_OP_ATAN2: --sp; st[sp - 1] = atan2(st[sp - 1], st[sp]); break;
      case SGH_OP_NEG: st[sp - 1] = -st[sp - 1]; break;
      case SGH_OP_SQRT: st[sp - 1] = sqrt(st[sp - 1]); break;
      case SGH_OP_EXP: st[sp - 1] = exp(st[sp - 1]); break;
      case SGH_OP_LOG: st[sp - 1] = log(st[sp - 1]); break;
      case SGH_OP_LOG2: st[sp - 1] = log2(st[sp - 1]); break;
      case SGH_OP_LOG10: st[sp - 1] = log10(st[sp - 1]); break;
      case SGH_OP_SIN: st[sp - 1] = sin(st[sp - 1]); break;
      case SGH_OP_COS: st[sp - 1] = cos(st[sp - 1]); break;
      case SGH_OP_TAN: st[sp - 1] = tan(st[sp - 1]); break;
      case SGH_OP_ASIN: st[sp - 1] = asin(st[sp - 1]); break;
      case SGH_OP_ACOS: st[sp - 1] = acos(st[sp - 1]); break;
      case SGH_OP_ATAN: st[sp - 1] = atan(st[sp - 1]); break;
      case SGH_OP_SINH: st[sp - 1] = sinh(st[sp - 1]); break;
      case SGH_OP_COSH: st[sp - 1] = cosh(st[sp - 1]); break;
      case SGH_OP_TANH: st[sp - 1] = tanh(st[sp - 1]); break;
      case SGH_OP_ASINH: st[sp - 1] = asinh(st[sp - 1]); break;
      case SGH_OP_ACOSH: st[sp - 1] = acosh(st[sp - 1]); break;
      case SGH_OP_ATANH: st[sp - 1] = atanh(st[sp - 1]); break;
      case SGH_OP_FABS: st[sp - 1] = fabs(st[sp - 1]); break;
      case SGH_OP_CEIL: st[sp - 1] = ceil(st[sp - 1]); break;
      case SGH_OP_FLOOR: st[sp - 1] = floor(st[sp - 1]); break;
      case SGH_OP_TRUNC: st[sp - 1] = trunc(st[sp - 1]); break;
      case SGH_OP_LOG1P: st[sp - 1] = log1p(st[sp - 1]); break;
      case SGH_OP_EXPM1: st[sp - 1] = expm1(st[sp - 1]); break;
      default: return nan("");
    }
  }
  return sp > 0 ? st[0] : nan("");
}

// Load of an epilogue input that no thread writes during the kernel, through
// the read-only path. Written as non-volatile inline asm without a memory
// clobber, so the compiler may issue it ahead of earlier stores to other
// arrays (with a plain load it must assume they alias and serialise). Only
// for arrays that stay unwritten for the whole kernel; a load guarded by a
// bounds test stays behind the test (inline asm is not speculated).
__device__ __forceinline__ double ld_in(const double* p) {
  double v;
  asm("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// Pointwise constants of the step, held by value inside the axis-pass
// epilogues: kernel parameters, which the epilogues' global stores cannot
// alias, so the compiler keeps them in registers instead of reloading
// DevParams after every store. Non-affine property programs are read
// through `full`.
// A modal value as a plan stores it: FP64, or rounded to FP32 in
// mixed-precision plans (the FP32 modal state of the mixed form).
__device__ __forceinline__ double st_mode(double x, int round32) { return round32 ? (double)(float)x : x; }

struct PointPhys {
  int nz, S, latent_model, degenerate_band, k_constant, has_top_conv, round32;
  int affine[P_COUNT];
  double sqrt_dV, omega, T_solidus, T_liquidus, band_inv, latent_factor, L_f, inv_dt;
  double kbar, abar, T0, h_top, T_boil, evap_f1, evap_f2, recon_scale;
  double aff_a[P_COUNT], aff_b[P_COUNT];
  const DevParams* full;
};

// Built on the host from the host copy of the parameters and the device copy.
inline PointPhys point_phys(const DevParams& h, const DevParams* dev) {
  PointPhys q;
  q.nz = h.nz; q.S = h.S; q.latent_model = h.latent_model; q.degenerate_band = h.degenerate_band;
  q.k_constant = h.k_constant; q.has_top_conv = h.has_top_conv; q.round32 = h.round32;
  for (int i = 0; i < P_COUNT; ++i) {
    q.affine[i] = h.affine[i];
    q.aff_a[i] = h.aff_a[i];
    q.aff_b[i] = h.aff_b[i];
  }
  q.sqrt_dV = h.sqrt_dV; q.omega = h.omega; q.T_solidus = h.T_solidus; q.T_liquidus = h.T_liquidus;
  q.band_inv = h.band_inv; q.latent_factor = h.latent_factor; q.L_f = h.L_f; q.inv_dt = h.inv_dt;
  q.kbar = h.kbar; q.abar = h.abar; q.T0 = h.T0; q.h_top = h.h_top; q.T_boil = h.T_boil;
  q.evap_f1 = h.evap_f1; q.evap_f2 = h.evap_f2; q.recon_scale = h.recon_scale;
  q.full = dev;
  return q;
}

__device__ __forceinline__ const sgh_program& prog_of(const DevParams& P, int slot) { return P.prog[slot]; }
__device__ __forceinline__ const sgh_program& prog_of(const PointPhys& P, int slot) { return P.full->prog[slot]; }

// One property branch: affine programs (the common piecewise-linear tables)
// take one FMA; anything else runs the postfix interpreter.
template <class PP>
__device__ __forceinline__ double prop(const PP& P, int slot, double T) {
  if (P.affine[slot]) return fma(P.aff_b[slot], T, P.aff_a[slot]);
  return eval_program(prog_of(P, slot), T);
}

// Liquid fraction as the fused kernels compute it: clip((T - T_s) * inv, 0, 1),
// a step at T_s for a degenerate band (core/properties.py:175-183, 218-229).
template <class PP>
__device__ __forceinline__ double fl_kernel(const PP& P, double T) {
  if (P.degenerate_band) return T >= P.T_solidus ? 1.0 : 0.0;
  double f = (T - P.T_solidus) * P.band_inv;
  return f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
}

// k(T) as TempProperty.__call__ evaluates it (core/properties.py:96-103,
// liquid_fraction :61-77 by division).
template <class PP>
__device__ __forceinline__ double k_blended(const PP& P, double T) {
  const double ks = prop(P, P_K_SOLID, T);
  if (P.k_constant) return ks;
  const double kl = prop(P, P_K_LIQUID, T);
  double fl;
  if (P.degenerate_band) {
    fl = T >= P.T_solidus ? 1.0 : 0.0;
  } else {
    fl = (T - P.T_solidus) / (P.T_liquidus - P.T_solidus);
    fl = fl < 0.0 ? 0.0 : (fl > 1.0 ? 1.0 : fl);
  }
  return (1.0 - fl) * ks + fl * kl;
}

// k'(T) = k(T) - kbar of the fused kernel (core/properties.py:185-191).
template <class PP>
__device__ __forceinline__ double k_prime(const PP& P, double T) {
  const double fl = fl_kernel(P, T);
  const double om = 1.0 - fl;
  const double kv = om * prop(P, P_K_SOLID, T) + fl * prop(P, P_K_LIQUID, T);
  return kv - P.kbar;
}

// a'(T) = rho(T) c(T) - abar (core/properties.py:188-192).
template <class PP>
__device__ __forceinline__ double a_prime(const PP& P, double T) {
  const double fl = fl_kernel(P, T);
  const double om = 1.0 - fl;
  const double rv = om * prop(P, P_RHO_SOLID, T) + fl * prop(P, P_RHO_LIQUID, T);
  const double cv = om * prop(P, P_C_SOLID, T) + fl * prop(P, P_C_LIQUID, T);
  return rv * cv - P.abar;
}

// Latent sink Q = -rho(T) L_f (f_l(T) - f_l(T_prev)) / dt: blended-rho form
// (core/properties.py:212-236) or constant form
// (physics/spectral_cpu_kernels.py:115-140).
template <class PP>
__device__ __forceinline__ double latent_source(const PP& P, double T, double Tp) {
  if (P.latent_model) {
    const double flc = fl_kernel(P, T);
    const double flp = fl_kernel(P, Tp);
    const double om = 1.0 - flc;
    const double rho = om * prop(P, P_RHO_SOLID, T) + flc * prop(P, P_RHO_LIQUID, T);
    return -rho * P.L_f * (flc - flp) * P.inv_dt;
  }
  double fc = (T - P.T_solidus) * P.band_inv;
  fc = fc < 0.0 ? 0.0 : (fc > 1.0 ? 1.0 : fc);
  double fp = (Tp - P.T_solidus) * P.band_inv;
  fp = fp < 0.0 ? 0.0 : (fp > 1.0 ? 1.0 : fp);
  return P.latent_factor * (fc - fp);
}

// Evaporation flux (physics/spectral_cpu_kernels.py:144-162). PP is any
// parameter block with T_liquidus, T_boil, evap_f1, evap_f2.
template <class PP>
__device__ __forceinline__ double evaporation(const PP& P, double T) {
  if (T < P.T_liquidus) return 0.0;
  const double term = (1.0 / sqrt(T)) * exp(P.evap_f2 * (1.0 - P.T_boil / T));
  return P.evap_f1 * term;
}

// Laser flux at cell (x, y) (core/laser.py:42-53 point-sampled super-Gaussian,
// :65-91 cell-integrated Gaussian). PP is any parameter block with dx, dy,
// r_x, r_y, order, cell_integrated.
template <class PP>
__device__ __forceinline__ double laser_flux(const PP& P, double I0, double x0, double y0,
                                             double x, double y) {
  if (P.cell_integrated) {
    const double s2 = sqrt(2.0);
    const double hx = P.dx, hy = P.dy;
    const double nxm = P.r_x * sqrt(M_PI / 8.0);
    const double nym = P.r_y * sqrt(M_PI / 8.0);
    const double ax = (x - x0 - hx / 2.0) * s2 / P.r_x;
    const double bx = (x - x0 + hx / 2.0) * s2 / P.r_x;
    const double ay = (y - y0 - hy / 2.0) * s2 / P.r_y;
    const double by = (y - y0 + hy / 2.0) * s2 / P.r_y;
    const double mx = nxm * (erf(bx) - erf(ax)) / hx;
    const double my = nym * (erf(by) - erf(ay)) / hy;
    return I0 * (my * mx);
  }
  const double ux = (x - x0) / P.r_x;
  const double uy = (y - y0) / P.r_y;
  const double r2 = ux * ux + uy * uy;
  const double shape = (P.order == 2.0) ? exp(-2.0 * r2) : exp(-2.0 * pow(r2, P.order / 2.0));
  return I0 * shape;
}

// Shift v*dt/d in cells of size d. A float32 laser state (SGH_LASER_F32,
// G-code paths) has the reference form it in float32: the product with a
// Python float dt and the quotient by a Python float d both round to float32
// (solvers/spectral.py:303-305, physics/spectral_cpu_kernels.py:392-396).
__device__ __forceinline__ double laser_shift(double v, double dt, double d, bool f32) {
  if (f32) return (double)__fdiv_rn(__fmul_rn((float)v, (float)dt), (float)d);
  return (v * dt) / d;
}

// Position in cells, x/d (physics/spectral_helpers.py:74), float32 for a
// float32 laser state.
__device__ __forceinline__ double laser_cells(double x, double d, bool f32) {
  if (f32) return (double)__fdiv_rn((float)x, (float)d);
  return x / d;
}

// Order-1 shift table entry for output index o (physics/spectral_cpu_kernels.py:305-325).
struct ShiftTap {
  int i0, i1;
  double w0, w1;
  bool in;
};
__device__ __forceinline__ ShiftTap shift_tap(int o, int n, double shift) {
  const double p = (double)o - shift;
  const double fl = floor(p);
  const double t = p - fl;
  ShiftTap s;
  s.in = (p >= 0.0) && (p <= (double)(n - 1));
  long long i0 = (long long)fl;
  long long i1 = i0 + 1;
  s.i0 = (int)(i0 < 0 ? 0 : (i0 > n - 1 ? n - 1 : i0));
  s.i1 = (int)(i1 < 0 ? 0 : (i1 > n - 1 ? n - 1 : i1));
  s.w1 = t;
  s.w0 = 1.0 - t;
  return s;
}

// ---------------------------------------------------------------------------
// block reductions (deterministic: fixed shuffle tree, then warp 0)
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void block_sum2(double& a, double& b, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) { sh[2 * w] = a; sh[2 * w + 1] = b; }
  __syncthreads();
  if (w == 0) {
    a = lane < NT / 32 ? sh[2 * lane] : 0.0;
    b = lane < NT / 32 ? sh[2 * lane + 1] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
  }
}

template <int NT>
__device__ __forceinline__ void block_max_sum(double& m, double& s, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    s += __shfl_down_sync(0xffffffffu, s, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) { sh[2 * w] = m; sh[2 * w + 1] = s; }
  __syncthreads();
  if (w == 0) {
    m = lane < NT / 32 ? sh[2 * lane] : -INFINITY;
    s = lane < NT / 32 ? sh[2 * lane + 1] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
      s += __shfl_down_sync(0xffffffffu, s, o);
    }
  }
}

// Error reporting shared by the library's translation units (sgh_last_error).
int set_error(int code, const char* msg);

}  // namespace sgh
