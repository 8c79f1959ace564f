// sgh_outputs.cu -- output reconstruction of a modal field on the device.
//
// The reference reconstructs outputs on the host after copying the modes out
// (physics/spectral_helpers.py): the node-centred volume field of every
// full-volume output (reconstruct_temperature_DCT, :146-204), and point
// values along the temperature profiles (reconstruct_temperature_volume_at_points,
// :206-248, used by save_temp_profiles, :251-333). Here both run on the modes
// where they live:
//
// * the node-centred field T[z_l][y_k][x_j] = sum a[p][n][m] C_m cos(m pi j / Nx)
//   C_n cos(n pi k / Ny) C_p cos(p pi l / Nz), j = 0..Nx (likewise k, l), as
//   three axis passes (sgh_axis.cuh) with (N+1) x N node cosine matrices --
//   the same cosine series the reference evaluates as a weighted DCT-I;
// * values at arbitrary points, T_i = sum a[p][n][m] Bz[p][i] By[n][i] Bx[m][i]
//   with B[m][i] = C_m cos(pi m x_i / L) on coordinates clipped to the domain,
//   as a contraction over 32-point tiles (one point per lane, warps over the
//   (p, n) rows of the modes).
//
// C_0 = sqrt(1/L), C_m = sqrt(2/L) (physics/spectral_helpers.py:26-46). FP64
// throughout. Every kernel indexes only inside the buffers whose sizes the
// entry points check; nothing waits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "sgh_b200.h"
#include "sgh_axis.cuh"
#include "sgh_device.cuh"

namespace sgh {
namespace outputs {

constexpr int T = 256;

// B[j][m] = C_m cos(pi m j / N), j = 0..N, m < N; the argument is reduced
// exactly in integers (cos(pi m j / N) has period 2N in m j).
__global__ void k_node_matrix(int N, double L, double* B) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)(N + 1) * N) return;
  const int j = (int)(e / N), m = (int)(e - (long long)j * N);
  const long long r = ((long long)m * j) % (2LL * N);
  const double c = (m == 0) ? sqrt(1.0 / L) : sqrt(2.0 / L);
  B[e] = c * cospi((double)r / (double)N);
}

// B[m][i] = C_m cos(pi m x_i / L), x_i = coords[3 i + col] clipped to [0, L]
// (spectral_helpers.py:87-106 and :235-237).
__global__ void k_point_basis(int n_modes, double L, int n, const double* coords, int col, double* B) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n_modes * n) return;
  const int m = (int)(e / n), i = (int)(e - (long long)m * n);
  const double x = fmin(fmax(coords[3LL * i + col], 0.0), L);
  const double c = (m == 0) ? sqrt(1.0 / L) : sqrt(2.0 / L);
  B[e] = c * cos(M_PI * (double)m * x / L);
}

// T_i for 32 points per CTA: lane = point, warp w takes rows r = w, w + 8, ...
// of the nz * ny rows; the row's x-sum is weighted by By and Bz of the point.
__global__ void __launch_bounds__(T) k_points(int nx, int ny, int nz, const double* a, int n, const double* Bx,
                                              const double* By, const double* Bz, double* out) {
  __shared__ double part[T / 32][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  const bool valid = i < n;
  double acc = 0.0;
  for (int r = warp; r < nz * ny; r += T / 32) {
    const int p = r / ny, q = r - p * ny;
    const double* row = a + (size_t)r * nx;
    double s = 0.0;
    for (int m = 0; m < nx; ++m) s = fma(__ldg(row + m), valid ? Bx[(size_t)m * n + i] : 0.0, s);
    if (valid) acc = fma(s, By[(size_t)q * n + i] * Bz[(size_t)p * n + i], acc);
  }
  part[warp][lane] = acc;
  __syncthreads();
  if (warp == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < T / 32; ++w) t += part[w][lane];
    if (valid) out[i] = t;
  }
}

// w[m] = C_m cos(pi m u / L), u = clip(pos, 0, L): the basis of one axis at
// one position (a fixed coordinate of a profile line).
__global__ void k_axis_weights(int n_modes, double L, double pos, double* w) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_modes) return;
  const double u = fmin(fmax(pos, 0.0), L);
  const double c = (m == 0) ? sqrt(1.0 / L) : sqrt(2.0 / L);
  w[m] = c * cos(M_PI * (double)m * u / L);
}

// T_i = sum_k A[k] C_k cos(pi k x_i / L) for points x_i (clipped) along one
// axis: the cosine series of the line, one point per thread.
__global__ void k_line_eval(int n_modes, double L, const double* A, int n, const double* x, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double u = fmin(fmax(x[i], 0.0), L);
  double t = 0.0;
  for (int k = 0; k < n_modes; ++k) {
    const double c = (k == 0) ? sqrt(1.0 / L) : sqrt(2.0 / L);
    t = fma(A[k], c * cos(M_PI * (double)k * u / L), t);
  }
  out[i] = t;
}

inline int blocks(long long n) { return (int)((n + T - 1) / T); }

size_t line_bytes(int nx, int ny, int nz) {
  const size_t w = (size_t)nx + ny + nz;
  const size_t t = std::max((size_t)nx * ny, (size_t)nz * ny);
  return sizeof(double) * (w + t + (size_t)std::max(nx, std::max(ny, nz)));
}

inline bool axes_ok(int nx, int ny, int nz) {
  return nx >= 1 && ny >= 1 && nz >= 1 && nx <= 4096 && ny <= 4096 && nz <= 4096;
}

int check_shape(int nx, int ny, int nz, double Lx, double Ly, double Lz) {
  if (!axes_ok(nx, ny, nz)) return set_error(SGH_ERR_INVALID, "axis lengths must be in [1, 4096]");
  if ((long long)(nx + 1) * (ny + 1) * (nz + 1) > (1LL << 30))
    return set_error(SGH_ERR_INVALID, "node grid exceeds 2^30 points");
  if (!(Lx > 0 && Ly > 0 && Lz > 0)) return set_error(SGH_ERR_INVALID, "domain lengths must be positive");
  return SGH_OK;
}

size_t nodal_bytes(int nx, int ny, int nz) {
  const size_t mats = (size_t)(nx + 1) * nx + (size_t)(ny + 1) * ny + (size_t)(nz + 1) * nz;
  const size_t tmp = (size_t)nz * (ny + 1) * (nx + 1);
  return sizeof(double) * (mats + tmp);
}

size_t points_bytes(int nx, int ny, int nz, int n) {
  return sizeof(double) * (size_t)n * (size_t)(nx + ny + nz);
}

}  // namespace outputs
}  // namespace sgh

using namespace sgh;

extern "C" {

int sgh_nodal_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, uint64_t* bytes) {
  if (!bytes) return set_error(SGH_ERR_INVALID, "null argument");
  if (!outputs::axes_ok(nx, ny, nz)) return set_error(SGH_ERR_INVALID, "axis lengths must be in [1, 4096]");
  *bytes = outputs::nodal_bytes(nx, ny, nz);
  return SGH_OK;
}

int sgh_nodal_temperature(int32_t nx, int32_t ny, int32_t nz, double Lx, double Ly, double Lz,
                          const double* modes, double* out, void* workspace, uint64_t bytes, void* stream) {
  const int rc = outputs::check_shape(nx, ny, nz, Lx, Ly, Lz);
  if (rc) return rc;
  if (!modes || !out || !workspace) return set_error(SGH_ERR_INVALID, "null pointer");
  if (bytes < outputs::nodal_bytes(nx, ny, nz))
    return set_error(SGH_ERR_WORKSPACE, "workspace smaller than sgh_nodal_workspace_bytes()");
  if ((const void*)modes == (const void*)out) return set_error(SGH_ERR_INVALID, "modes and out must differ");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* Bx = static_cast<double*>(workspace);
  double* By = Bx + (size_t)(nx + 1) * nx;
  double* Bz = By + (size_t)(ny + 1) * ny;
  double* tmp = Bz + (size_t)(nz + 1) * nz;
  outputs::k_node_matrix<<<outputs::blocks((long long)(nx + 1) * nx), outputs::T, 0, s>>>(nx, Lx, Bx);
  outputs::k_node_matrix<<<outputs::blocks((long long)(ny + 1) * ny), outputs::T, 0, s>>>(ny, Ly, By);
  outputs::k_node_matrix<<<outputs::blocks((long long)(nz + 1) * nz), outputs::T, 0, s>>>(nz, Lz, Bz);
  // x: modes (nz, ny, nx) -> out as (nz, ny, nx+1); y: -> tmp (nz, ny+1, nx+1);
  // z: tmp -> out (nz+1, ny+1, nx+1). The first result fits in out: nz ny (nx+1) <= (nz+1)(ny+1)(nx+1).
  launch_axis(modes, Bx, nx + 1, nx, nz * ny, 1, EpiStore{out, 1.0, nullptr}, s);
  launch_axis(out, By, ny + 1, ny, nz, nx + 1, EpiStore{tmp, 1.0, nullptr}, s);
  launch_axis(tmp, Bz, nz + 1, nz, 1, (ny + 1) * (nx + 1), EpiStore{out, 1.0, nullptr}, s);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SGH_ERR_CUDA, cudaGetErrorString(e));
  return SGH_OK;
}

int sgh_points_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, int32_t n_points, uint64_t* bytes) {
  if (!bytes) return set_error(SGH_ERR_INVALID, "null argument");
  if (!outputs::axes_ok(nx, ny, nz) || n_points < 0)
    return set_error(SGH_ERR_INVALID, "axis lengths must be in [1, 4096] and n_points >= 0");
  *bytes = outputs::points_bytes(nx, ny, nz, n_points);
  return SGH_OK;
}

int sgh_points_temperature(int32_t nx, int32_t ny, int32_t nz, double Lx, double Ly, double Lz,
                           const double* modes, int32_t n_points, const double* coords, double* out,
                           void* workspace, uint64_t bytes, void* stream) {
  const int rc = outputs::check_shape(nx, ny, nz, Lx, Ly, Lz);
  if (rc) return rc;
  if (n_points < 0) return set_error(SGH_ERR_INVALID, "n_points must be >= 0");
  if (n_points == 0) return SGH_OK;
  if (!modes || !coords || !out || !workspace) return set_error(SGH_ERR_INVALID, "null pointer");
  if (bytes < outputs::points_bytes(nx, ny, nz, n_points))
    return set_error(SGH_ERR_WORKSPACE, "workspace smaller than sgh_points_workspace_bytes()");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* Bx = static_cast<double*>(workspace);
  double* By = Bx + (size_t)nx * n_points;
  double* Bz = By + (size_t)ny * n_points;
  outputs::k_point_basis<<<outputs::blocks((long long)nx * n_points), outputs::T, 0, s>>>(nx, Lx, n_points, coords, 0, Bx);
  outputs::k_point_basis<<<outputs::blocks((long long)ny * n_points), outputs::T, 0, s>>>(ny, Ly, n_points, coords, 1, By);
  outputs::k_point_basis<<<outputs::blocks((long long)nz * n_points), outputs::T, 0, s>>>(nz, Lz, n_points, coords, 2, Bz);
  outputs::k_points<<<(n_points + 31) / 32, outputs::T, 0, s>>>(nx, ny, nz, modes, n_points, Bx, By, Bz, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SGH_ERR_CUDA, cudaGetErrorString(e));
  return SGH_OK;
}

int sgh_line_workspace_bytes(int32_t nx, int32_t ny, int32_t nz, uint64_t* bytes) {
  if (!bytes) return set_error(SGH_ERR_INVALID, "null argument");
  if (!outputs::axes_ok(nx, ny, nz)) return set_error(SGH_ERR_INVALID, "axis lengths must be in [1, 4096]");
  *bytes = outputs::line_bytes(nx, ny, nz);
  return SGH_OK;
}

int sgh_line_temperature(int32_t nx, int32_t ny, int32_t nz, double Lx, double Ly, double Lz,
                         const double* modes, int32_t axis, double x, double y, double z, int32_t n_points,
                         const double* coords, double* out, void* workspace, uint64_t bytes, void* stream) {
  const int rc = outputs::check_shape(nx, ny, nz, Lx, Ly, Lz);
  if (rc) return rc;
  if (axis < 0 || axis > 2) return set_error(SGH_ERR_INVALID, "axis must be 0 (x), 1 (y) or 2 (z)");
  if (n_points < 0) return set_error(SGH_ERR_INVALID, "n_points must be >= 0");
  if (n_points == 0) return SGH_OK;
  if (!modes || !coords || !out || !workspace) return set_error(SGH_ERR_INVALID, "null pointer");
  if (bytes < outputs::line_bytes(nx, ny, nz))
    return set_error(SGH_ERR_WORKSPACE, "workspace smaller than sgh_line_workspace_bytes()");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* wx = static_cast<double*>(workspace);
  double* wy = wx + nx;
  double* wz = wy + ny;
  double* t1 = wz + nz;
  double* A = t1 + std::max((size_t)nx * ny, (size_t)nz * ny);
  const int S = nx * ny;
  // weights of the two fixed axes, then two one-row axis passes that reduce
  // the modes to the series of the line (largest reduction first)
  if (axis == 0) {
    outputs::k_axis_weights<<<outputs::blocks(ny), outputs::T, 0, s>>>(ny, Ly, y, wy);
    outputs::k_axis_weights<<<outputs::blocks(nz), outputs::T, 0, s>>>(nz, Lz, z, wz);
    launch_axis(modes, wz, 1, nz, 1, S, EpiStore{t1, 1.0, nullptr}, s);   // (ny, nx)
    launch_axis(t1, wy, 1, ny, 1, nx, EpiStore{A, 1.0, nullptr}, s);      // (nx)
    outputs::k_line_eval<<<outputs::blocks(n_points), outputs::T, 0, s>>>(nx, Lx, A, n_points, coords, out);
  } else if (axis == 1) {
    outputs::k_axis_weights<<<outputs::blocks(nx), outputs::T, 0, s>>>(nx, Lx, x, wx);
    outputs::k_axis_weights<<<outputs::blocks(nz), outputs::T, 0, s>>>(nz, Lz, z, wz);
    launch_axis(modes, wz, 1, nz, 1, S, EpiStore{t1, 1.0, nullptr}, s);   // (ny, nx)
    launch_axis(t1, wx, 1, nx, ny, 1, EpiStore{A, 1.0, nullptr}, s);      // (ny)
    outputs::k_line_eval<<<outputs::blocks(n_points), outputs::T, 0, s>>>(ny, Ly, A, n_points, coords, out);
  } else {
    outputs::k_axis_weights<<<outputs::blocks(nx), outputs::T, 0, s>>>(nx, Lx, x, wx);
    outputs::k_axis_weights<<<outputs::blocks(ny), outputs::T, 0, s>>>(ny, Ly, y, wy);
    launch_axis(modes, wx, 1, nx, nz * ny, 1, EpiStore{t1, 1.0, nullptr}, s);  // (nz, ny)
    launch_axis(t1, wy, 1, ny, nz, 1, EpiStore{A, 1.0, nullptr}, s);           // (nz)
    outputs::k_line_eval<<<outputs::blocks(n_points), outputs::T, 0, s>>>(nz, Lz, A, n_points, coords, out);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SGH_ERR_CUDA, cudaGetErrorString(e));
  return SGH_OK;
}

}  // extern "C"
