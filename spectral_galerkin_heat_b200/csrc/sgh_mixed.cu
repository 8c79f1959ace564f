// sgh_mixed.cu -- split-BF16 tensor-core DCT contractions (tcgen05).
//
// sgh_dct2_bf16x3: orthonormal 2-D DCT-II / DCT-III of an (ny, nx) face with
// both passes on the tensor cores in split-BF16 form (three products per
// k-step, FP32 accumulation in tensor memory); FP64 in and out. This is the
// face contraction of the mixed-precision step.
#include <cuda_runtime.h>

#include <string>

#include "sgh_b200.h"
#include "sgh_device.cuh"
#include "sgh_umma.cuh"

namespace sgh {
namespace mixed {

struct LoadRowMajor {  // value(r, k) = p[r * ld + k]
  const double* p;
  int ld;
  __device__ __forceinline__ double operator()(int r, int k) const { return p[(size_t)r * ld + k]; }
};
struct LoadColMajor {  // value(r, k) = p[k * ld + r]
  const double* p;
  int ld;
  __device__ __forceinline__ double operator()(int r, int k) const { return p[(size_t)k * ld + r]; }
};
struct StoreRowMajor {
  double* p;
  int ld;
  __device__ __forceinline__ void operator()(int m, int n, double v) const { p[(size_t)m * ld + n] = v; }
};

// PASS 0: out[y][k] = sum_n in[y][n] Mx[k][n]   (M = ny, N = nx, K = nx)
// PASS 1: out[k][x] = sum_n My[k][n] in[n][x]   (M = ny, N = nx, K = ny)
template <int NT, int PASS>
__global__ void __launch_bounds__(umma::THREADS)
k_dct2_bf16x3(const double* in, double* out, const double* Mx, const double* My, int ny, int nx, int* err) {
  extern __shared__ __align__(128) char smem[];
  const int m0 = blockIdx.y * umma::TM, n0 = blockIdx.x * NT;
  if (PASS == 0)
    umma::tile_bf16x3<NT>(ny, nx, nx, m0, n0, LoadRowMajor{in, nx}, LoadRowMajor{Mx, nx}, StoreRowMajor{out, nx},
                          smem, err);
  else
    umma::tile_bf16x3<NT>(ny, nx, ny, m0, n0, LoadRowMajor{My, ny}, LoadColMajor{in, nx}, StoreRowMajor{out, nx},
                          smem, err);
}

__global__ void k_dct_matrix_mixed(int N, double* M) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * N) return;
  const int k = e / N, n = e - k * N;
  const long long m = ((long long)k * (2 * n + 1)) % (4LL * N);
  const double w = (k == 0) ? sqrt(1.0 / N) : sqrt(2.0 / N);
  const double v = w * cospi((double)m / (double)(2 * N));
  M[k * N + n] = v;
  M[(size_t)N * N + n * N + k] = v;
}

template <int NT, int PASS>
int launch_pass(const double* in, double* out, const double* Mx, const double* My, int ny, int nx, int* err,
                cudaStream_t s) {
  const int smem = umma::smem_bytes(NT);
  cudaError_t e = cudaFuncSetAttribute(k_dct2_bf16x3<NT, PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return set_error(SGH_ERR_CUDA, cudaGetErrorString(e));
  dim3 grid((nx + NT - 1) / NT, (ny + umma::TM - 1) / umma::TM);
  k_dct2_bf16x3<NT, PASS><<<grid, umma::THREADS, smem, s>>>(in, out, Mx, My, ny, nx, err);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SGH_ERR_CUDA, cudaGetErrorString(e));
  return SGH_OK;
}

template <int PASS>
int launch_nt(const double* in, double* out, const double* Mx, const double* My, int ny, int nx, int* err,
              cudaStream_t s) {
  if (nx <= 64) return launch_pass<64, PASS>(in, out, Mx, My, ny, nx, err, s);
  if (nx <= 128) return launch_pass<128, PASS>(in, out, Mx, My, ny, nx, err, s);
  return launch_pass<256, PASS>(in, out, Mx, My, ny, nx, err, s);
}

struct Dct2Layout {
  size_t o_err = 0, o_mx = 0, o_my = 0, o_t = 0, total = 0;
};
inline size_t take(size_t& off, size_t bytes) {
  const size_t o = off;
  off += (bytes + 255) & ~size_t(255);
  return o;
}
inline Dct2Layout dct2_layout(int ny, int nx) {
  Dct2Layout L;
  size_t off = 0;
  L.o_err = take(off, 256);
  L.o_mx = take(off, sizeof(double) * 2 * (size_t)nx * nx);
  L.o_my = take(off, sizeof(double) * 2 * (size_t)ny * ny);
  L.o_t = take(off, sizeof(double) * (size_t)nx * ny);
  L.total = off;
  return L;
}

}  // namespace mixed
}  // namespace sgh

using namespace sgh;
using namespace sgh::mixed;

extern "C" {

int sgh_dct2_bf16x3_workspace_bytes(int32_t ny, int32_t nx, uint64_t* bytes) {
  if (!bytes) return set_error(SGH_ERR_INVALID, "null argument");
  if (ny < 1 || nx < 1 || ny > 4096 || nx > 4096) return set_error(SGH_ERR_INVALID, "face axes must be in [1, 4096]");
  *bytes = dct2_layout(ny, nx).total;
  return SGH_OK;
}

int sgh_dct2_bf16x3(int32_t kind, int32_t ny, int32_t nx, const double* in, double* out, void* workspace,
                    uint64_t bytes, void* stream) {
  if (!in || !out || !workspace) return set_error(SGH_ERR_INVALID, "null argument");
  if (kind != 2 && kind != 3) return set_error(SGH_ERR_INVALID, "kind must be 2 (DCT_II) or 3 (IDCT_II)");
  if (ny < 1 || nx < 1 || ny > 4096 || nx > 4096) return set_error(SGH_ERR_INVALID, "face axes must be in [1, 4096]");
  const Dct2Layout L = dct2_layout(ny, nx);
  if (bytes < L.total) return set_error(SGH_ERR_WORKSPACE, "workspace is smaller than sgh_dct2_bf16x3_workspace_bytes()");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return set_error(SGH_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* ws = static_cast<char*>(workspace);
  int* err = reinterpret_cast<int*>(ws + L.o_err);
  double* Mx = reinterpret_cast<double*>(ws + L.o_mx);
  double* My = reinterpret_cast<double*>(ws + L.o_my);
  double* t = reinterpret_cast<double*>(ws + L.o_t);
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
  if (e != cudaSuccess) return set_error(SGH_ERR_CUDA, cudaGetErrorString(e));
  k_dct_matrix_mixed<<<(nx * nx + 255) / 256, 256, 0, s>>>(nx, Mx);
  k_dct_matrix_mixed<<<(ny * ny + 255) / 256, 256, 0, s>>>(ny, My);
  const size_t offx = (kind == 3) ? (size_t)nx * nx : 0, offy = (kind == 3) ? (size_t)ny * ny : 0;
  int rc = launch_nt<0>(in, t, Mx + offx, My + offy, ny, nx, err, s);
  if (rc) return rc;
  rc = launch_nt<1>(t, out, Mx + offx, My + offy, ny, nx, err, s);
  return rc;
}

}  // extern "C"
