// Exhaustive check of spectral_rs_b200/csrc/exact_math.cuh against the IEEE
// round-to-nearest reciprocal and square root: every float in [1, 2^126) for the
// fast paths, and special values (0, subnormals, below 1, 2^126 and above, inf,
// NaN, negatives) for the guarded versions.  Prints the mismatch counts; exits 1
// on any mismatch.  Built and run by tests/test_gpu_rounding.py.
#include <cstdio>
#include <cstring>

#include "exact_math.cuh"

__device__ bool same(float a, float b) {  // bitwise, NaNs of any payload equal
  return __float_as_uint(a) == __float_as_uint(b) || (a != a && b != b);
}

__global__ void k_domain(unsigned long long lo, unsigned long long hi, unsigned long long* bad, unsigned* first) {
  for (unsigned long long b = lo + blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; b < hi;
       b += (unsigned long long)gridDim.x * blockDim.x) {
    const float x = __uint_as_float((unsigned)b);
    if (!same(spx::rcp_rn_ge1(x), __frcp_rn(x))) {
      atomicAdd(&bad[0], 1ull);
      atomicMin(&first[0], (unsigned)b);
    }
    if (!same(spx::sqrt_rn_ge1(x), __fsqrt_rn(x))) {
      atomicAdd(&bad[1], 1ull);
      atomicMin(&first[1], (unsigned)b);
    }
  }
}

__global__ void k_special(const float* xs, int n, unsigned long long* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = xs[i];
  if (!same(spx::rcp_exact(x), __frcp_rn(x))) atomicAdd(&bad[2], 1ull);
  if (!same(spx::sqrt_exact(x), __fsqrt_rn(x))) atomicAdd(&bad[3], 1ull);
}

static float f_of(unsigned u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

int main() {
  unsigned long long* bad;
  unsigned* first;
  float* xs;
  cudaMallocManaged(&bad, 4 * sizeof(unsigned long long));
  cudaMallocManaged(&first, 2 * sizeof(unsigned));
  const float sp[] = {0.0f, -0.0f, f_of(1u), f_of(0x007FFFFFu), f_of(0x00800000u), 1e-30f, 0.5f, 0.999999940f,
                      1.0f, 1.00000012f, 3.0f, f_of(0x7E7FFFFFu), f_of(0x7E800000u), f_of(0x7F7FFFFFu),
                      f_of(0x7F800000u), f_of(0x7FC00000u), -1.0f, -3.0f, f_of(0xFF800000u)};
  const int nsp = sizeof(sp) / sizeof(sp[0]);
  cudaMallocManaged(&xs, sizeof(sp));
  std::memcpy(xs, sp, sizeof(sp));
  bad[0] = bad[1] = bad[2] = bad[3] = 0;
  first[0] = first[1] = 0xFFFFFFFFu;
  k_domain<<<148 * 16, 256>>>(0x3F800000ull, 0x7E800000ull, bad, first);  // [1, 2^126)
  k_special<<<1, 64>>>(xs, nsp, bad);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    std::printf("cuda error: %s\n", cudaGetErrorString(e));
    return 2;
  }
  std::printf("rcp mismatches %llu (first 0x%08x), sqrt mismatches %llu (first 0x%08x), "
              "guarded specials: rcp %llu, sqrt %llu\n",
              bad[0], first[0], bad[1], first[1], bad[2], bad[3]);
  return (bad[0] | bad[1] | bad[2] | bad[3]) ? 1 : 0;
}
