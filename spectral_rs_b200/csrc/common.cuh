// Shared definitions of the B200 hot-path library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/spectral_gpu.h"

namespace spx {

// ----------------------------------------------------------------------------
// Host-side error plumbing: every device call is checked and turned into a
// status code plus a message kept on the context.
// ----------------------------------------------------------------------------
struct Status {
  int code = SPX_OK;
  std::string msg;
};

#define SPX_CUDA_TRY(call)                                                              \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess) {                                                            \
      throw ::spx::Error(SPX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    }                                                                                   \
  } while (0)

struct Error {
  int code;
  std::string msg;
  Error(int c, std::string m) : code(c), msg(std::move(m)) {}
};

// ----------------------------------------------------------------------------
// Grid geometry in the reference layout.
//   spatial: (ny+2) x (nx+2) floats, row-major, ghost frame at row/col 0 and n+1
//   spectral: ny x nx float2, row-major (ky rows, kx columns); the field update
//   keeps the half spectrum of its real fields, ny x nx/2 (kx in [0, nx/2))
// ----------------------------------------------------------------------------
struct Grid {
  int nx, ny;      // interior cells
  int W;           // nx + 2, spatial row pitch
  int log2nx, log2ny;
  __host__ __device__ int sidx(int row, int col) const { return row * W + col; }
  __host__ __device__ size_t spatial_size() const { return (size_t)(ny + 2) * (size_t)W; }
  __host__ __device__ size_t spectral_size() const { return (size_t)ny * (size_t)nx; }
  __host__ __device__ size_t half_spectral_size() const { return (size_t)ny * (size_t)(nx / 2); }
};

// Wave numbers restated from src/flds/wave_num.rs:18-33 in FP32 with the same
// operation order, so on-the-fly values equal the reference's table bit for bit.
__host__ __device__ inline float wave_kx(int j, int n) {
  const float PI = 3.14159265358979323846f;
  float k = (float)j;
  if (j >= n / 2 + 1) k -= (float)n;
  k *= 2.0f * PI / (float)n;  // (2*PI)/n, then one rounding multiply
  return k;
}

}  // namespace spx
