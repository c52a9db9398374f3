// Pseudo-spectral Maxwell solver on the B200 (replaces src/flds/*.rs of the reference).
//
// Data layout in HBM
//   spatial fields: reference layout, (ny+2) x (nx+2) floats with a one-cell ghost frame
//   spectral fields: half spectra, ny x nx/2 float2, row-major (ky rows, kx in [0, nx/2)),
//   numpy fft2 convention; the other half is the conjugate mirror (the fields are real)
//   and column nx/2 is zero after every update
//
// Kernels per Flds::update (src/flds/mod.rs:87-309):
//   k_filter_fused         : n_pass 3x3 binomial passes of jx, jy, jz, dsty
//   k_rows_r2c             : copy_to_spectral (+ dsty * 1/dens) fused with the row FFTs of
//                            7 fields, two real rows per complex transform
//   k_cols<fwd>            : column FFTs of the 7 half spectra, strip of W columns per CTA
//   k_kspace               : Ampere, divergence correction, Faraday, Nyquist, B average
//   k_cols<inv>            : column inverse FFTs of B(t) and E
//   k_rows_c2r             : row inverse FFTs (two real rows per transform), 1/(nx ny)
//                            scale, copy_to_spatial + update_ghosts fused
//
// The FFT is a Stockham autosort transform (radix 8 passes, one radix 4 or 2
// pass for the remaining factor), one radix-8 butterfly per thread per pass:
// the first pass reads global memory into registers, the last one writes from
// registers, the passes in between exchange through shared memory; twiddles
// from an FP64-generated table.  Inverse transforms use
// ifft(x) = conj(fft(conj(x))), conjugating on load and store.
#include <cmath>
#include <vector>

#include <cstring>

#include "fields.cuh"

namespace spx {

bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }
int ilog2(uint64_t v) {
  int l = 0;
  while ((1ull << l) < v) ++l;
  return l;
}

void make_twiddles(int n, float2* out) {
  // exp(-2 pi i m / n) evaluated in long double, using the octant symmetries so
  // that every entry is the correctly rounded value of an exact-angle sin/cos.
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    long double a = two_pi * (long double)m / (long double)n;
    long double c = cosl(a), s = sinl(a);
    if (4 * m == n) { c = 0; s = 1; }
    if (2 * m == n) { c = -1; s = 0; }
    if (4 * m == 3 * n) { c = 0; s = -1; }
    if (m == 0) { c = 1; s = 0; }
    out[m] = make_float2((float)(double)c, (float)(double)(-s));
  }
}

// Pass-major twiddle records.  Every pass after the first (Ns = 8^p earlier
// outputs per group, radix R) has Ns records of R float2 (8 for radix 8):
// record k holds w^(r k step), r = 1 .. R-1, step = n / (Ns R), then one unused
// slot, so a butterfly reads its twiddles as R/2 aligned 16-byte loads.  The
// values are entries of make_twiddles(n).
static int host_passes(int logN) { return logN / 3 + (logN % 3 ? 1 : 0); }
static int host_last_radix(int logN) { return logN % 3 == 0 ? 8 : (logN % 3 == 2 ? 4 : 2); }
size_t pass_twiddle_count(int n) {
  const int logN = ilog2(n), np = host_passes(logN);
  size_t total = 0;
  for (int i = 1, logNs = 3; i < np; ++i, logNs += 3) total += ((size_t)1 << logNs) * (i < np - 1 ? 8 : host_last_radix(logN));
  return std::max<size_t>(total, 2);
}
std::vector<float2> make_pass_twiddles(int n) {
  std::vector<float2> tw(n), out(pass_twiddle_count(n), make_float2(0.f, 0.f));
  make_twiddles(n, tw.data());
  const int logN = ilog2(n), np = host_passes(logN);
  size_t base = 0;
  for (int i = 1, logNs = 3; i < np; ++i, logNs += 3) {
    const int R = i < np - 1 ? 8 : host_last_radix(logN);
    const int Ns = 1 << logNs, step = n / (Ns * R);
    for (int k = 0; k < Ns; ++k)
      for (int r = 1; r < R; ++r) out[base + (size_t)k * R + (r - 1)] = tw[(size_t)r * k * step];
    base += (size_t)Ns * R;
  }
  return out;
}

// ---------------------------------------------------------------- complex
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// ---------------------------------------------------------------- radix kernels (forward)
__device__ __forceinline__ void dft2(float2& a, float2& b) {
  float2 t = a;
  a = c_add(t, b);
  b = c_sub(t, b);
}
__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
  float2 t0 = c_add(v0, v2), t1 = c_sub(v0, v2), t2 = c_add(v1, v3), t3 = c_sub(v1, v3);
  t3 = make_float2(t3.y, -t3.x);  // -i * (v1 - v3)
  v0 = c_add(t0, t2);
  v2 = c_sub(t0, t2);
  v1 = c_add(t1, t3);
  v3 = c_sub(t1, t3);
}
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3);
  dft4(o0, o1, o2, o3);
  const float r = 0.70710678118654752440f;  // 1/sqrt(2): W8 = (1 - i)/sqrt(2)
  float2 w1 = make_float2((o1.x + o1.y) * r, (o1.y - o1.x) * r);
  float2 w2 = make_float2(o2.y, -o2.x);
  float2 w3 = make_float2((o3.y - o3.x) * r, -(o3.x + o3.y) * r);
  v[0] = c_add(e0, o0);
  v[4] = c_sub(e0, o0);
  v[1] = c_add(e1, w1);
  v[5] = c_sub(e1, w1);
  v[2] = c_add(e2, w2);
  v[6] = c_sub(e2, w2);
  v[3] = c_add(e3, w3);
  v[7] = c_sub(e3, w3);
}

// Stockham passes over B = 2^logB transforms of length N = 2^logN with
// blockDim.x == N*B/8: pass p of radix R has each thread do 8/R butterflies
// b = tid + q*blockDim.x, each on transform t and index j in [0, N/R), with
// inputs at positions j + r*N/R and outputs at ((j - k)*R + k) + r*Ns, k = j mod
// Ns (Ns = product of the earlier radices).  The first pass (radix 8) takes its
// inputs from registers and the last pass leaves its outputs in registers, so
// the caller loads and stores global memory directly; the passes in between
// exchange through shared memory, element (t, e) at s[pad(t*TS + e*ES)] with
// one padding slot per 16 elements against bank conflicts.  Radix 8 passes,
// then one radix 4 or 2 pass for the remaining factor.
__device__ __forceinline__ int spad(int i) { return i + (i >> 4); }
__host__ __device__ inline size_t fft_smem_elems(int logN, int logB) {
  const size_t n = (size_t)1 << (logN + logB);
  return n + (n >> 4) + 1;
}
__device__ __forceinline__ int num_passes(int logN) { return logN / 3 + (logN % 3 ? 1 : 0); }
__device__ __forceinline__ int last_radix(int logN) { return logN % 3 == 0 ? 8 : (logN % 3 == 2 ? 4 : 2); }

template <int R>
__device__ __forceinline__ void bfly_tj(int q, int logN, int logB, bool t_fast, int& t, int& j) {
  constexpr int LR = R == 8 ? 3 : R == 4 ? 2 : 1;
  const int b = threadIdx.x + q * blockDim.x;
  const int logNb = logN - LR;
  if (t_fast) {
    t = b & ((1 << logB) - 1);
    j = b >> logB;
  } else {
    t = b >> logNb;
    j = b & ((1 << logNb) - 1);
  }
}

// twiddles and DFTs of the thread's butterflies, slot q*R + r = input r of butterfly q;
// Ns = 2^logNs (all index arithmetic is on powers of two: shifts and masks);
// twp: this pass's twiddle records (make_pass_twiddles)
template <int R>
__device__ __forceinline__ void pass_compute(float2 (&v)[8], int logN, int logB, bool t_fast, int logNs,
                                             const float2* __restrict__ twp) {
  constexpr int PER = 8 / R;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    if (logNs > 0) {
      int t, j;
      bfly_tj<R>(q, logN, logB, t_fast, t, j);
      const int k = j & ((1 << logNs) - 1);
      const float4* rec = reinterpret_cast<const float4*>(twp + (size_t)k * R);
      float2 w[R];
#pragma unroll
      for (int l = 0; l < R / 2; ++l) {
        const float4 p = __ldg(rec + l);
        w[2 * l] = make_float2(p.x, p.y);
        w[2 * l + 1] = make_float2(p.z, p.w);
      }
#pragma unroll
      for (int r = 1; r < R; ++r) v[q * R + r] = c_mul(v[q * R + r], w[r - 1]);
    }
    if constexpr (R == 8) {
      dft8(v);
    } else if constexpr (R == 4) {
      dft4(v[q * 4 + 0], v[q * 4 + 1], v[q * 4 + 2], v[q * 4 + 3]);
    } else {
      dft2(v[q * 2 + 0], v[q * 2 + 1]);
    }
  }
}

template <int R>
__device__ __forceinline__ void pass_store(const float2 (&v)[8], float2* s, int logN, int logB, int ES, int TS,
                                           bool t_fast, int logNs) {
  constexpr int PER = 8 / R;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    int t, j;
    bfly_tj<R>(q, logN, logB, t_fast, t, j);
    const int k = j & ((1 << logNs) - 1);
    const int base = t * TS + ((j - k) * R + k) * ES;
#pragma unroll
    for (int r = 0; r < R; ++r) s[spad(base + ((r * ES) << logNs))] = v[q * R + r];
  }
}

template <int R>
__device__ __forceinline__ void pass_load(float2 (&v)[8], const float2* s, int logN, int logB, int ES, int TS,
                                          bool t_fast) {
  constexpr int PER = 8 / R;
  constexpr int LR = R == 8 ? 3 : R == 4 ? 2 : 1;
  const int nb = (1 << logN) >> LR;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    int t, j;
    bfly_tj<R>(q, logN, logB, t_fast, t, j);
#pragma unroll
    for (int r = 0; r < R; ++r) v[q * R + r] = s[spad(t * TS + (j + r * nb) * ES)];
  }
}

// Forward FFT.  On entry v[r] = element (t, j + r*N/8) with (t, j) = bfly_tj<8>(0);
// on exit v[m] = element out_pos(m).
__device__ __forceinline__ void block_fft_regs(float2 (&v)[8], float2* s, int logN, int logB, int ES, int TS,
                                               bool t_fast, const float2* __restrict__ tw) {
  const int np = num_passes(logN);
  pass_compute<8>(v, logN, logB, t_fast, 0, tw);
  int logNs = 0;
  const float2* twp = tw;  // records of the current pass
  for (int i = 1; i < np; ++i) {
    pass_store<8>(v, s, logN, logB, ES, TS, t_fast, logNs);  // only the last pass can have radix < 8
    __syncthreads();
    if (i > 1) twp += (size_t)8 << logNs;  // the previous pass had radix 8
    logNs += 3;
    const int R = (i < np - 1) ? 8 : last_radix(logN);
    if (R == 8) {
      pass_load<8>(v, s, logN, logB, ES, TS, t_fast);
      pass_compute<8>(v, logN, logB, t_fast, logNs, twp);
    } else if (R == 4) {
      pass_load<4>(v, s, logN, logB, ES, TS, t_fast);
      pass_compute<4>(v, logN, logB, t_fast, logNs, twp);
    } else {
      pass_load<2>(v, s, logN, logB, ES, TS, t_fast);
      pass_compute<2>(v, logN, logB, t_fast, logNs, twp);
    }
    __syncthreads();  // every thread has read before the next pass overwrites
  }
}

// Position of output slot m after block_fft_regs: last pass radix R = last_radix,
// butterfly q = m / R, r = m % R, e = j + r*N/R (k = j in the last pass).
__device__ __forceinline__ void out_pos(int m, int logN, int logB, bool t_fast, int& t, int& e) {
  const int R = num_passes(logN) == 1 ? 8 : last_radix(logN);
  const int LR = R == 8 ? 3 : R == 4 ? 2 : 1;
  const int q = m >> LR, r = m & (R - 1);
  int j;
  if (R == 8)
    bfly_tj<8>(q, logN, logB, t_fast, t, j);
  else if (R == 4)
    bfly_tj<4>(q, logN, logB, t_fast, t, j);
  else
    bfly_tj<2>(q, logN, logB, t_fast, t, j);
  e = j + (r << (logN - LR));
}

// ---------------------------------------------------------------- launch geometry
// Row pass: B rows per CTA with blockDim = N*B/8 threads.
__host__ __device__ constexpr int row_logB(int logN) {
  int lb = 11 - logN;  // N*B = 2048 -> 256 threads for small rows
  return lb < 0 ? 0 : lb;
}
// Column pass: strip of W = 2^logW columns, blockDim = Ny*W/8 threads (<= 1024).
// 512 threads (two CTAs per SM at 64 registers) while the strip is at least 4
// columns (32-byte row segments), else 1024 threads; >= 256 for short columns.
__host__ __device__ inline int col_logW(int logNy, int logNx) {
  int lw = logNy >= 7 ? 12 - logNy : 11 - logNy;
  if (logNy >= 7 && lw < 2) lw = 13 - logNy;
  if (lw > 4 && logNy >= 7) lw = 4;  // 16 columns = 128 B row segments
  if (lw < 0) lw = 0;
  if (lw > logNx) lw = logNx;
  return lw;
}

// ---------------------------------------------------------------- row kernels
// The spatial fields are real, so each field's 2-D spectrum is Hermitian,
// F[ky][nx - kx] = conj F[ny - ky][kx], and the update zeroes column kx = nx/2
// (src/flds/mod.rs:230-266).  The field update therefore keeps the spectra of
// columns kx in [0, nx/2) only (the "half spectrum", ny x nx/2 complex), and
// its row transforms carry two real rows of a field in one complex FFT:
//   forward  z = a + i b, Z = fft(z): A[k] = (Z[k] + conj Z[-k]) / 2,
//                                     B[k] = (Z[k] - conj Z[-k]) / (2i);
//   inverse  Z[k] = A[k] + i B[k] (negative k from conj A, conj B), z = ifft(Z):
//            a = Re z, b = Im z.
// The reference transforms each real field as a complex one (im = 0,
// src/flds/field.rs:78-139) and keeps Re of the inverse; the pairing computes
// the same DFT with half the transforms, so results agree to FP32 rounding.
struct RowArgs {
  const void* src[8];
  void* dst[8];
  float* back[8];  // forward: when set, the input value is also stored here (ghosted, periodic ghosts)
  float scale[8];
};

// Store the value of interior cell (row, e) (0-based) into a ghosted spatial
// field together with the ghost cells that are its periodic images
// (copy_to_spatial followed by update_ghosts, src/flds/field.rs:128-257).
__device__ __forceinline__ void store_ghosted(float* dst, const Grid& g, int row, int e, float v) {
  const int N = g.nx, W = g.W;
  const int R = row + 1;  // ghosted row
  dst[(size_t)R * W + e + 1] = v;
  if (e == N - 1) dst[(size_t)R * W + 0] = v;  // left ghost <- last column
  if (e == 0) dst[(size_t)R * W + N + 1] = v;  // right ghost <- first column
  if (R == g.ny) {                             // top ghost row <- last row
    dst[e + 1] = v;
    if (e == N - 1) dst[0] = v;      // top-left <- bottom-right
    if (e == 0) dst[N + 1] = v;      // top-right <- bottom-left
  }
  if (R == 1) {  // bottom ghost row <- first row
    dst[(size_t)(g.ny + 1) * W + e + 1] = v;
    if (e == N - 1) dst[(size_t)(g.ny + 1) * W + 0] = v;      // bottom-left <- top-right
    if (e == 0) dst[(size_t)(g.ny + 1) * W + N + 1] = v;      // bottom-right <- top-left
  }
}

// Launch bounds of the transforms: a launch of at most 512 threads (every
// transform of <= 4096 points) runs the SMALL instantiation, bounded to three
// such CTAs per SM (40 registers); 8192-point transforms need 1024 threads.
#define FFT_BOUNDS(SMALL) __launch_bounds__((SMALL) ? 512 : 1024, (SMALL) ? 3 : 1)
// LOGN > 0: the transform length 2^LOGN as a compile-time constant (every index
// of the passes folds); LOGN = 0 reads it from the grid.
constexpr int FFT_LOGN_MIN = 6, FFT_LOGN_MAX = 13;

// Complex row FFTs of full ny x nx arrays (Fft2D on a complex array, the tests'
// path): CTA = B = 2^row_logB rows of one field.
template <bool INV, bool SMALL, int LOGN>
__global__ void FFT_BOUNDS(SMALL) k_rows(const __grid_constant__ RowArgs a, Grid g0, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  Grid g = g0;
  if (LOGN) {
    g.log2nx = LOGN;
    g.nx = 1 << LOGN;
    g.W = g.nx + 2;
  }
  const int f = blockIdx.y;
  const int logN = g.log2nx, N = g.nx;
  const int logB = row_logB(logN);
  const int row0 = blockIdx.x << logB;
  const float sc = a.scale[f];
  float2 v[8];
  {
    int t, j;
    bfly_tj<8>(0, logN, logB, false, t, j);
    const int row = row0 + t;
    const float2* __restrict__ src = (const float2*)a.src[f];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const float2 x = row < g.ny ? src[(size_t)row * N + j + r * (N >> 3)] : make_float2(0.f, 0.f);
      v[r] = INV ? c_conj(x) : x;
    }
  }
  block_fft_regs(v, sm, logN, logB, 1, N, false, tw);
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    int t, e;
    out_pos(m, logN, logB, false, t, e);
    const int row = row0 + t;
    if (row >= g.ny) continue;
    float2 x = v[m];
    if (INV) x = c_conj(x);
    ((float2*)a.dst[f])[(size_t)row * N + e] = INV ? c_scale(x, sc) : x;
  }
}

// Forward row transforms of real ghosted fields into half spectra (copy_to_spectral
// fused, src/flds/field.rs:78-106): CTA = B = 2^row_logB pairs of rows (2p, 2p+1)
// of field blockIdx.y, one complex FFT per pair.  a.scale multiplies the input
// (1/dens for dsty, src/flds/mod.rs:66-85).
template <bool SMALL, int LOGN>
__global__ void FFT_BOUNDS(SMALL) k_rows_r2c(const __grid_constant__ RowArgs a0, const RowArgs* __restrict__ tab,
                                             Grid g0, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const RowArgs& a = tab ? tab[blockIdx.z] : a0;  // a batch: member blockIdx.z's fields
  Grid g = g0;
  if (LOGN) {
    g.log2nx = LOGN;
    g.nx = 1 << LOGN;
    g.W = g.nx + 2;
  }
  const int f = blockIdx.y;
  const int logN = g.log2nx, N = g.nx, H = N >> 1;
  const int logB = row_logB(logN);
  const int p0 = blockIdx.x << logB, npairs = g.ny >> 1;
  const float sc = a.scale[f];
  float2 v[8];
  {
    int t, j;
    bfly_tj<8>(0, logN, logB, false, t, j);
    const int p = p0 + t;
    const float* __restrict__ src = (const float*)a.src[f];
    // all 16 loads first, then the write-back stores (which may not be reordered above them)
    float u0[8], u1[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const size_t o = (size_t)(2 * p + 1) * g.W + j + r * (N >> 3) + 1;
      u0[r] = p < npairs ? src[o] : 0.f;
      u1[r] = p < npairs ? src[o + g.W] : 0.f;
    }
    if (a.back[f] && p < npairs)
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        store_ghosted(a.back[f], g, 2 * p, j + r * (N >> 3), u0[r]);
        store_ghosted(a.back[f], g, 2 * p + 1, j + r * (N >> 3), u1[r]);
      }
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = make_float2(u0[r] * sc, u1[r] * sc);
  }
  block_fft_regs(v, sm, logN, logB, 1, N, false, tw);  // ends with a barrier after the last reads
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    int t, e;
    out_pos(m, logN, logB, false, t, e);
    sm[spad(t * N + e)] = v[m];
  }
  __syncthreads();
  // unpack: (pair t, k < N/2), four per thread, consecutive k on consecutive threads
  float2* __restrict__ dst = (float2*)a.dst[f];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int b = threadIdx.x + q * blockDim.x;
    const int t = b >> (logN - 1), k = b & (H - 1);
    const int p = p0 + t;
    const float2 zk = sm[spad(t * N + k)], zm = sm[spad(t * N + ((N - k) & (N - 1)))];
    if (p < npairs) {
      dst[(size_t)(2 * p) * H + k] = make_float2((zk.x + zm.x) * 0.5f, (zk.y - zm.y) * 0.5f);
      dst[(size_t)(2 * p + 1) * H + k] = make_float2((zk.y + zm.y) * 0.5f, (zm.x - zk.x) * 0.5f);
    }
  }
}

// Inverse row transforms of half spectra into real ghosted fields (copy_to_spatial
// and update_ghosts fused, src/flds/field.rs:108-257): pairs of rows as above;
// a.scale = 1/(nx ny) (src/flds/fft_2d.rs:170-171).
template <bool SMALL, int LOGN>
__global__ void FFT_BOUNDS(SMALL) k_rows_c2r(const __grid_constant__ RowArgs a0, const RowArgs* __restrict__ tab,
                                             Grid g0, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const RowArgs& a = tab ? tab[blockIdx.z] : a0;
  Grid g = g0;
  if (LOGN) {
    g.log2nx = LOGN;
    g.nx = 1 << LOGN;
    g.W = g.nx + 2;
  }
  const int f = blockIdx.y;
  const int logN = g.log2nx, N = g.nx, H = N >> 1;
  const int logB = row_logB(logN);
  const int p0 = blockIdx.x << logB, npairs = g.ny >> 1;
  const float sc = a.scale[f];
  float2 v[8];
  {
    int t, j;
    bfly_tj<8>(0, logN, logB, false, t, j);
    const int p = p0 + t;
    const float2* __restrict__ s0 = (const float2*)a.src[f] + (size_t)(2 * p) * H;
    const float2* __restrict__ s1 = s0 + H;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      // inputs r < 4 lie in [0, N/2), inputs r >= 4 in [N/2, N): their conjugate partners
      const int e = j + r * (N >> 3);
      const int k = r < 4 ? e : (N - e) & (N - 1);
      float2 z = make_float2(0.f, 0.f);
      if (p < npairs && (r < 4 || e != H)) {  // column N/2 is zero
        const float2 x = s0[k], y = s1[k];
        z = r < 4 ? make_float2(x.x - y.y, x.y + y.x)   // A + i B
                  : make_float2(x.x + y.y, y.x - x.y);  // conj A + i conj B
      }
      v[r] = c_conj(z);  // inverse as conj(fft(conj(Z)))
    }
  }
  block_fft_regs(v, sm, logN, logB, 1, N, false, tw);
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    int t, e;
    out_pos(m, logN, logB, false, t, e);
    const int p = p0 + t;
    if (p >= npairs) continue;
    // Re and Im of the inverse (the conjugation of the result flips only Im)
    store_ghosted((float*)a.dst[f], g, 2 * p, e, v[m].x * sc);
    store_ghosted((float*)a.dst[f], g, 2 * p + 1, e, -v[m].y * sc);
  }
}

// Column FFTs, in place on complex arrays: CTA = strip of W columns of one field.
struct ColArgs {
  float2* data[8];
};
template <bool INV, bool SMALL, int LOGN>
__global__ void FFT_BOUNDS(SMALL) k_cols(const __grid_constant__ ColArgs a0, const ColArgs* __restrict__ tab, Grid g0,
                                         const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const ColArgs& a = tab ? tab[blockIdx.z] : a0;
  Grid g = g0;
  if (LOGN) {
    g.log2ny = LOGN;
    g.ny = 1 << LOGN;
  }
  const int f = blockIdx.y;
  const int logN = g.log2ny, N = g.ny;
  const int logW = col_logW(g.log2ny, g.log2nx);
  const int W = 1 << logW;
  const int x0 = blockIdx.x << logW;
  float2* d = a.data[f];
  float2 v[8];
  {
    int t, j;
    bfly_tj<8>(0, logN, logW, true, t, j);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const float2 x = d[(size_t)(j + r * (N >> 3)) * g.nx + x0 + t];
      v[r] = INV ? c_conj(x) : x;
    }
  }
  block_fft_regs(v, sm, logN, logW, W, 1, true, tw);
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    int t, y;
    out_pos(m, logN, logW, true, t, y);
    d[(size_t)y * g.nx + x0 + t] = INV ? c_conj(v[m]) : v[m];
  }
}

// ---------------------------------------------------------------- k-space update
// src/flds/mod.rs:105-278 for one k point; num_complex operation order.  Over the
// half spectrum (kx = j in [0, nx/2), ny x nx/2 points): the update is pointwise
// and maps a Hermitian spectrum to a Hermitian one, and it zeroes column nx/2.
struct KArgs {
  float2 *jx, *jy, *jz, *rho, *ex, *ey, *ez, *bwx, *bwy, *bwz, *bax, *bay, *baz;
  float cdt, ckc;
};
__global__ void k_kspace(const __grid_constant__ KArgs a0, const KArgs* __restrict__ tab, Grid g) {
  const KArgs& a = tab ? tab[blockIdx.y] : a0;
  const size_t n = g.half_spectral_size();
  const int logH = g.log2nx - 1;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx >> logH), j = (int)(idx & ((1 << logH) - 1));
    const float kx = wave_kx(j, g.nx), ky = wave_kx(i, g.ny);
    float2 Jx = a.jx[idx], Jy = a.jy[idx], Jz = a.jz[idx], Rho = a.rho[idx];
    if (idx == 0) {  // mod.rs:106-107 (j_z[0] is not zeroed)
      Jx = make_float2(0.f, 0.f);
      Jy = make_float2(0.f, 0.f);
    }
    const float2 Bx = a.bwx[idx], By = a.bwy[idx], Bz = a.bwz[idx];  // b_*.spectral <- b_*_wrk (t-1/2)
    float2 Ex = a.ex[idx], Ey = a.ey[idx], Ez = a.ez[idx];
    const float cdt = a.cdt, ckc = a.ckc;
    // Ampere (mod.rs:130-173)
    Ex = c_add(Ex, c_sub(c_mul(make_float2(0.0f * ky, cdt * ky), Bz), make_float2(ckc * Jx.x, ckc * Jx.y)));
    Ey = c_add(Ey, c_sub(c_mul(make_float2(0.0f * kx, -cdt * kx), Bz), make_float2(ckc * Jy.x, ckc * Jy.y)));
    {
      float2 kb = c_sub(make_float2(kx * By.x, kx * By.y), make_float2(ky * Bx.x, ky * Bx.y));
      Ez = c_add(Ez, c_mul(make_float2(0.0f, cdt), kb));
      Ez = c_sub(Ez, make_float2(ckc * Jz.x, ckc * Jz.y));
    }
    // divergence correction with k_norm = 1/k^2, k = 0 kept (mod.rs:177-207)
    if (idx != 0) {
      const float kn = 1.0f / (kx * kx + ky * ky);
      float2 t = c_add(c_add(make_float2(kx * Ex.x, kx * Ex.y), make_float2(ky * Ey.x, ky * Ey.y)),
                       c_mul(make_float2(0.f, 1.f), Rho));
      t = c_scale(t, kn);
      Ex = c_sub(Ex, c_scale(t, kx));
      Ey = c_sub(Ey, c_scale(t, ky));
    }
    // Faraday to t+1/2 (mod.rs:211-225)
    float2 nBx = c_sub(Bx, c_mul(make_float2(0.0f * ky, cdt * ky), Ez));
    float2 nBy = c_add(By, c_mul(make_float2(0.0f * kx, cdt * kx), Ez));
    float2 nBz = c_add(Bz, c_mul(make_float2(0.0f, cdt),
                                 c_sub(make_float2(ky * Ex.x, ky * Ex.y), make_float2(kx * Ey.x, kx * Ey.y))));
    // Nyquist row ky = ny/2 (mod.rs:230-266); column kx = nx/2 is not stored
    if (i == g.ny / 2) {
      const float2 z = make_float2(0.f, 0.f);
      nBx = nBy = nBz = z;
      Ex = Ey = Ez = z;
    }
    a.ex[idx] = Ex;
    a.ey[idx] = Ey;
    a.ez[idx] = Ez;
    a.bwx[idx] = nBx;
    a.bwy[idx] = nBy;
    a.bwz[idx] = nBz;
    // B at integer time (mod.rs:270-278)
    a.bax[idx] = c_scale(c_add(Bx, nBx), 0.5f);
    a.bay[idx] = c_scale(c_add(By, nBy), 0.5f);
    a.baz[idx] = c_scale(c_add(Bz, nBz), 0.5f);
  }
}

// ---------------------------------------------------------------- ghost frame kernels
struct FieldList {
  float* f[SPX_NUM_FIELDS];
};
struct ConstFieldList {
  const float* f[SPX_NUM_FIELDS];
};

// Field::deposit_ghosts, one thread per interior cell of the frame; additions in
// the reference's order (rows, columns, corners), so results are bit-exact.
__global__ void k_fold(const __grid_constant__ FieldList L, const FieldList* __restrict__ tab, Grid g) {
  float* F = tab ? tab[blockIdx.z].f[blockIdx.y] : L.f[blockIdx.y];
  const int nx = g.nx, ny = g.ny, W = g.W;
  const int nper = 2 * nx + 2 * (ny - 2);
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nper; p += gridDim.x * blockDim.x) {
    int r, c;
    if (p < nx) { r = 1; c = p + 1; }
    else if (p < 2 * nx) { r = ny; c = p - nx + 1; }
    else if (p < 2 * nx + ny - 2) { r = p - 2 * nx + 2; c = 1; }
    else { r = p - 2 * nx - (ny - 2) + 2; c = nx; }
    float v = F[r * W + c];
    if (r == ny) v = __fadd_rn(v, F[0 * W + c]);
    if (r == 1) v = __fadd_rn(v, F[(ny + 1) * W + c]);
    if (c == nx) v = __fadd_rn(v, F[r * W + 0]);
    if (c == 1) v = __fadd_rn(v, F[r * W + nx + 1]);
    if (r == ny && c == nx) v = __fadd_rn(v, F[0]);
    if (r == ny && c == 1) v = __fadd_rn(v, F[nx + 1]);
    if (r == 1 && c == nx) v = __fadd_rn(v, F[(ny + 1) * W + 0]);
    if (r == 1 && c == 1) v = __fadd_rn(v, F[(ny + 1) * W + nx + 1]);
    F[r * W + c] = v;
  }
}

__device__ __forceinline__ int wrap_row(int r, int n) { return r == 0 ? n : (r == n + 1 ? 1 : r); }

// Field::update_ghosts: every ghost cell <- its periodic interior image.
__global__ void k_update_ghosts(const __grid_constant__ FieldList L, Grid g) {
  float* F = L.f[blockIdx.y];
  const int nx = g.nx, ny = g.ny, W = g.W;
  const int nper = 2 * (nx + 2) + 2 * ny;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nper; p += gridDim.x * blockDim.x) {
    int r, c;
    if (p < nx + 2) { r = 0; c = p; }
    else if (p < 2 * (nx + 2)) { r = ny + 1; c = p - (nx + 2); }
    else if (p < 2 * (nx + 2) + ny) { r = p - 2 * (nx + 2) + 1; c = 0; }
    else { r = p - 2 * (nx + 2) - ny + 1; c = nx + 1; }
    F[r * W + c] = F[wrap_row(r, ny) * W + wrap_row(c, nx)];
  }
}

// One binomial_filter_2_d pass for every cell of the ghosted output: interior
// cells apply the 1-2-1 x 1-2-1 / 16 stencil to the input (whose ghost cells
// hold whatever the input had, as in the reference); ghost cells receive the
// filtered value of their periodic image (the update_ghosts that follows in
// the reference).  Reference summation order, no contraction: bit-exact.
__global__ void k_filter(const __grid_constant__ ConstFieldList S, const __grid_constant__ FieldList D, Grid g) {
  const float* in = S.f[blockIdx.z];
  float* out = D.f[blockIdx.z];
  const int W = g.W;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  if (c > g.nx + 1 || r > g.ny + 1) return;
  const int ri = wrap_row(r, g.ny), ci = wrap_row(c, g.nx);
  const float* up = in + (ri - 1) * W + ci;
  const float* md = in + ri * W + ci;
  const float* dn = in + (ri + 1) * W + ci;
  float v = __fmul_rn(0.0625f, up[-1]);
  v = __fadd_rn(v, __fmul_rn(0.125f, up[0]));
  v = __fadd_rn(v, __fmul_rn(0.0625f, up[1]));
  v = __fadd_rn(v, __fmul_rn(0.125f, md[-1]));
  v = __fadd_rn(v, __fmul_rn(0.25f, md[0]));
  v = __fadd_rn(v, __fmul_rn(0.125f, md[1]));
  v = __fadd_rn(v, __fmul_rn(0.0625f, dn[-1]));
  v = __fadd_rn(v, __fmul_rn(0.125f, dn[0]));
  v = __fadd_rn(v, __fmul_rn(0.0625f, dn[1]));
  out[r * W + c] = v;
}

// Fused filter geometry: the extended frame of a tile is 64 columns wide (one
// per lane of a 64-thread row group; 4 row groups = 256 threads), the output
// tile is 64 - 2h columns by FILT_TY rows, h = n_pass - 1 (up to 15).
constexpr int FILT_EW = 64, FILT_TY = 32, FILT_MAX_PASS = 16;

// binomial_filter_2_d's stencil at the cell whose 3x3 neighbourhood rows start
// at up, md, dn (left column): reference summation order, no contraction.
__device__ __forceinline__ float binomial9(const float* up, const float* md, const float* dn) {
  float v = __fmul_rn(0.0625f, up[0]);
  v = __fadd_rn(v, __fmul_rn(0.125f, up[1]));
  v = __fadd_rn(v, __fmul_rn(0.0625f, up[2]));
  v = __fadd_rn(v, __fmul_rn(0.125f, md[0]));
  v = __fadd_rn(v, __fmul_rn(0.25f, md[1]));
  v = __fadd_rn(v, __fmul_rn(0.125f, md[2]));
  v = __fadd_rn(v, __fmul_rn(0.0625f, dn[0]));
  v = __fadd_rn(v, __fmul_rn(0.125f, dn[1]));
  v = __fadd_rn(v, __fmul_rn(0.0625f, dn[2]));
  return v;
}

// n passes of binomial_filter_2_d in one kernel (the reference runs them one
// after another, each followed by update_ghosts, src/flds/mod.rs:90-94).  Pass
// 1 reads the raw ghosted input around each cell's periodic image; after it
// every neighbour is a periodic image, so passes 2..n run on a shared-memory
// frame whose halo shrinks by one cell per pass.  Each lane owns one column of
// the frame and walks a chunk of rows keeping the last two rows of its 3x3
// neighbourhood in registers (3 shared loads per cell).  Writes the interior of
// `out`; each value is computed exactly as the separate passes compute it.
__host__ __device__ inline size_t filter_fused_smem_floats(int npass) {
  const int h = npass - 1;
  const size_t eh = FILT_TY + 2 * h;
  return 2 * (size_t)FILT_EW * eh + (FILT_EW + 2) * (eh + 2);
}

// One pass over frame rows [r0, r1) of column q (src row pitch sp; the 3x3
// neighbourhood of frame cell (r, q) is src[(r - 1 + dr) * sp + q - 1 + dq]).
__device__ __forceinline__ void filter_column(const float* src, int sp, float* dst, int dp, int q, int r0, int r1) {
  if (r0 >= r1) return;
  const float* s = src + q - 1;
  float a0 = s[(r0 - 1) * sp], a1 = s[(r0 - 1) * sp + 1], a2 = s[(r0 - 1) * sp + 2];
  float b0 = s[r0 * sp], b1 = s[r0 * sp + 1], b2 = s[r0 * sp + 2];
  for (int r = r0; r < r1; ++r) {
    const float c0 = s[(r + 1) * sp], c1 = s[(r + 1) * sp + 1], c2 = s[(r + 1) * sp + 2];
    const float up[3] = {a0, a1, a2}, md[3] = {b0, b1, b2}, dn[3] = {c0, c1, c2};
    dst[r * dp + q] = binomial9(up, md, dn);
    a0 = b0;
    a1 = b1;
    a2 = b2;
    b0 = c0;
    b1 = c1;
    b2 = c2;
  }
}

__global__ void __launch_bounds__(256) k_filter_fused(const __grid_constant__ ConstFieldList S,
                                                      const __grid_constant__ FieldList D,
                                                      const ConstFieldList* __restrict__ stab,
                                                      const FieldList* __restrict__ dtab, int nf, Grid g, int npass) {
  extern __shared__ float fs[];
  // a batch: blockIdx.z = member * nf + field
  const float* in = stab ? stab[blockIdx.z / nf].f[blockIdx.z % nf] : S.f[blockIdx.z];
  float* out = dtab ? dtab[blockIdx.z / nf].f[blockIdx.z % nf] : D.f[blockIdx.z];
  const int W = g.W, nx = g.nx, ny = g.ny;
  const int h = npass - 1;
  const int TW = FILT_EW - 2 * h;                // output tile width
  const int EW = FILT_EW, EH = FILT_TY + 2 * h;  // frame
  const int x0 = blockIdx.x * TW + 1, y0 = blockIdx.y * FILT_TY + 1;  // first interior cell of the tile
  const int ex0 = x0 - h, ey0 = y0 - h;                               // origin of the frame
  const int q = threadIdx.x & 63, grp = threadIdx.x >> 6;
  float* s0 = fs;
  float* s1 = fs + EW * EH;
  float* raw = fs + 2 * EW * EH;
  const bool inner = ex0 >= 1 && ey0 >= 1 && ex0 + EW - 1 <= nx && ey0 + EH - 1 <= ny;
  // rows [lo, hi) of a region split into 4 chunks, one per row group
  auto chunk = [&](int lo, int hi, int& r0, int& r1) {
    const int n = (hi - lo + 3) >> 2;
    r0 = min(hi, lo + grp * n);
    r1 = min(hi, r0 + n);
  };
  if (inner) {  // the frame and its one-cell border are plain array cells: raw (EW+2) x (EH+2)
    const int RW = EW + 2, RH = EH + 2;
    for (int r = grp; r < RH; r += 4) {
      const float* row = in + (size_t)(ey0 - 1 + r) * W + (ex0 - 1);
      raw[r * RW + q] = row[q];
      if (q < 2) raw[r * RW + 64 + q] = row[64 + q];
    }
    __syncthreads();
    int r0, r1;
    chunk(0, EH, r0, r1);
    filter_column(raw + RW + 1, RW, s0, EW, q, r0, r1);  // frame cell (r, q) = raw cell (r + 1, q + 1)
  } else {  // near the domain edge: the periodic image of each frame cell, raw ghosts included
    const int xx = (((ex0 + q - 1) % nx) + nx) % nx + 1;
    for (int r = grp; r < EH; r += 4) {
      const int yy = (((ey0 + r - 1) % ny) + ny) % ny + 1;
      const float* md = in + (size_t)yy * W + xx - 1;
      s0[r * EW + q] = binomial9(md - W, md, md + W);
    }
  }
  __syncthreads();
  float* src = s0;
  float* dst = s1;
  for (int p = 2; p <= npass; ++p) {
    const int m = p - 1;  // frame cells [m, EW - m) x [m, EH - m)
    int r0, r1;
    chunk(m, EH - m, r0, r1);
    if (q >= m && q < EW - m) filter_column(src, EW, dst, EW, q, r0, r1);
    __syncthreads();
    float* t = src;
    src = dst;
    dst = t;
  }
  if (q >= h && q < h + TW) {
    const int xx = x0 + q - h;
    if (xx <= nx)
      for (int r = grp; r < FILT_TY; r += 4) {
        const int yy = y0 + r;
        if (yy > ny) break;
        out[(size_t)yy * W + xx] = src[(r + h) * EW + q];
      }
  }
}

__global__ void k_scale_c(float2* d, size_t n, float s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = c_scale(d[i], s);
}

// ---------------------------------------------------------------- host launchers
void launch_fold(const Grid& g, float* const* fields, int nf, cudaStream_t st) {
  FieldList L{};
  for (int i = 0; i < nf; ++i) L.f[i] = fields[i];
  int nper = 2 * g.nx + 2 * (g.ny - 2);
  int blocks = (nper + 255) / 256;
  k_fold<<<dim3(blocks, nf), 256, 0, st>>>(L, nullptr, g);
}

void launch_update_ghosts(const Grid& g, float* const* fields, int nf, cudaStream_t st) {
  FieldList L{};
  for (int i = 0; i < nf; ++i) L.f[i] = fields[i];
  int nper = 2 * (g.nx + 2) + 2 * g.ny;
  k_update_ghosts<<<dim3((nper + 255) / 256, nf), 256, 0, st>>>(L, g);
}

bool filter_fused_fits(uint32_t npass) { return npass >= 1 && npass <= (uint32_t)FILT_MAX_PASS; }

void launch_filter_fused(const Grid& g, float* const* src, float* const* dst, int nf, uint32_t npass,
                         cudaStream_t st) {
  ConstFieldList S{};
  FieldList D{};
  for (int i = 0; i < nf; ++i) {
    S.f[i] = src[i];
    D.f[i] = dst[i];
  }
  const size_t smem = filter_fused_smem_floats((int)npass) * sizeof(float);
  const int tw = FILT_EW - 2 * ((int)npass - 1);
  dim3 grd((g.nx + tw - 1) / tw, (g.ny + FILT_TY - 1) / FILT_TY, nf);
  k_filter_fused<<<grd, 256, smem, st>>>(S, D, nullptr, nullptr, nf, g, (int)npass);
}

void launch_filter_pass(const Grid& g, float* const* src, float* const* dst, int nf, cudaStream_t st) {
  ConstFieldList S{};
  FieldList D{};
  for (int i = 0; i < nf; ++i) {
    S.f[i] = src[i];
    D.f[i] = dst[i];
  }
  dim3 blk(64, 4);
  dim3 grd((g.nx + 2 + 63) / 64, (g.ny + 2 + 3) / 4, nf);
  k_filter<<<grd, blk, 0, st>>>(S, D, g);
}

cudaError_t launch_filter_pass_status(const Grid& g, const float* src, float* dst, cudaStream_t st) {
  ConstFieldList S{};
  FieldList D{};
  S.f[0] = src;
  D.f[0] = dst;
  Grid gg = g;
  void* args[] = {&S, &D, &gg};
  const dim3 blk(64, 4);
  const dim3 grd((g.nx + 2 + 63) / 64, (g.ny + 2 + 3) / 4, 1);
  return cudaLaunchKernel((const void*)k_filter, grd, blk, args, 0, st);
}

// Dynamic shared memory above 48 KB must be opted into once per kernel (on
// every device that runs it; done when a context is created, never while a
// stream is being captured).
// Rows: the launch is SMALL when it has at most 512 threads, known at compile
// time for a given length.
constexpr bool rows_small(int logN) { return ((1 << logN) << row_logB(logN)) / 8 <= 512; }

static void fft_attr(const void* f) {
  SPX_CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
}
template <int LOGN>
static void fft_set_kernel_attributes() {
  if constexpr (LOGN == 0) {
    for (bool S : {true, false}) {
      fft_attr(S ? (const void*)k_rows<false, true, 0> : (const void*)k_rows<false, false, 0>);
      fft_attr(S ? (const void*)k_rows<true, true, 0> : (const void*)k_rows<true, false, 0>);
      fft_attr(S ? (const void*)k_rows_r2c<true, 0> : (const void*)k_rows_r2c<false, 0>);
      fft_attr(S ? (const void*)k_rows_c2r<true, 0> : (const void*)k_rows_c2r<false, 0>);
    }
  } else {
    constexpr bool S = rows_small(LOGN);
    fft_attr((const void*)k_rows<false, S, LOGN>);
    fft_attr((const void*)k_rows<true, S, LOGN>);
    fft_attr((const void*)k_rows_r2c<S, LOGN>);
    fft_attr((const void*)k_rows_c2r<S, LOGN>);
  }
  fft_attr((const void*)k_cols<false, true, LOGN>);
  fft_attr((const void*)k_cols<true, true, LOGN>);
  fft_attr((const void*)k_cols<false, false, LOGN>);
  fft_attr((const void*)k_cols<true, false, LOGN>);
  if constexpr (LOGN == 0)
    fft_set_kernel_attributes<FFT_LOGN_MIN>();
  else if constexpr (LOGN < FFT_LOGN_MAX)
    fft_set_kernel_attributes<LOGN + 1>();
}
void fields_set_kernel_attributes() {
  fft_set_kernel_attributes<0>();
  fft_attr((const void*)k_filter_fused);
}

// Complex row FFTs of a full array (tests).
template <bool INV, int LOGN>
static void launch_rows_n(const Grid& g, const RowArgs& a, int nf, const float2* tw, cudaStream_t st) {
  const int logB = row_logB(g.log2nx);
  const int threads = std::max(1, (g.nx << logB) / 8);
  const size_t smem = sizeof(float2) * fft_smem_elems(g.log2nx, logB);
  const int blocks = (g.ny + (1 << logB) - 1) >> logB;
  if constexpr (LOGN > 0) {
    k_rows<INV, rows_small(LOGN), LOGN><<<dim3(blocks, nf), threads, smem, st>>>(a, g, tw);
  } else {
    if (threads <= 512)
      k_rows<INV, true, 0><<<dim3(blocks, nf), threads, smem, st>>>(a, g, tw);
    else
      k_rows<INV, false, 0><<<dim3(blocks, nf), threads, smem, st>>>(a, g, tw);
  }
}

// Real-pair row transforms of the field update (forward r2c or inverse c2r);
// tab: a batch of nm simulations of grid g (member blockIdx.z's arguments), else a alone (nm = 1)
template <bool INV, int LOGN>
static void launch_pair_rows_n(const Grid& g, const RowArgs& a, const RowArgs* tab, int nf, int nm,
                               const float2* tw, cudaStream_t st) {
  const int logB = row_logB(g.log2nx);
  const int threads = std::max(1, (g.nx << logB) / 8);
  const size_t smem = sizeof(float2) * fft_smem_elems(g.log2nx, logB);
  const int blocks = ((g.ny >> 1) + (1 << logB) - 1) >> logB;
  const dim3 grid(blocks, nf, nm);
  if constexpr (LOGN > 0) {
    constexpr bool S = rows_small(LOGN);
    if (INV)
      k_rows_c2r<S, LOGN><<<grid, threads, smem, st>>>(a, tab, g, tw);
    else
      k_rows_r2c<S, LOGN><<<grid, threads, smem, st>>>(a, tab, g, tw);
  } else if (threads <= 512) {
    if (INV)
      k_rows_c2r<true, 0><<<grid, threads, smem, st>>>(a, tab, g, tw);
    else
      k_rows_r2c<true, 0><<<grid, threads, smem, st>>>(a, tab, g, tw);
  } else {
    if (INV)
      k_rows_c2r<false, 0><<<grid, threads, smem, st>>>(a, tab, g, tw);
    else
      k_rows_r2c<false, 0><<<grid, threads, smem, st>>>(a, tab, g, tw);
  }
}

// g: the grid of the columns (for the half spectra, half_grid of the simulation's)
template <bool INV, int LOGN>
static void launch_cols_n(const Grid& g, const ColArgs& a, const ColArgs* tab, int nf, int nm, const float2* tw,
                          cudaStream_t st) {
  const int logW = col_logW(g.log2ny, g.log2nx);
  const int threads = std::max(1, (g.ny << logW) / 8);
  const size_t smem = sizeof(float2) * fft_smem_elems(g.log2ny, logW);
  const int blocks = g.nx >> logW;
  if (threads <= 512)
    k_cols<INV, true, LOGN><<<dim3(blocks, nf, nm), threads, smem, st>>>(a, tab, g, tw);
  else
    k_cols<INV, false, LOGN><<<dim3(blocks, nf, nm), threads, smem, st>>>(a, tab, g, tw);
}

// Dispatch on the transform length: 2^6 .. 2^13 compiled per length, shorter ones generic.
#define FFT_DISPATCH(LOG, CALL) \
  switch (LOG) {                \
    case 6: CALL(6); break;     \
    case 7: CALL(7); break;     \
    case 8: CALL(8); break;     \
    case 9: CALL(9); break;     \
    case 10: CALL(10); break;   \
    case 11: CALL(11); break;   \
    case 12: CALL(12); break;   \
    case 13: CALL(13); break;   \
    default: CALL(0); break;    \
  }

template <bool INV>
static void launch_rows(const Grid& g, const RowArgs& a, int nf, const float2* tw, cudaStream_t st) {
#define SPX_ROWS(L) launch_rows_n<INV, L>(g, a, nf, tw, st)
  FFT_DISPATCH(g.log2nx, SPX_ROWS)
#undef SPX_ROWS
}

template <bool INV>
static void launch_pair_rows(const Grid& g, const RowArgs& a, int nf, const float2* tw, cudaStream_t st,
                             const RowArgs* tab = nullptr, int nm = 1) {
#define SPX_ROWS(L) launch_pair_rows_n<INV, L>(g, a, tab, nf, nm, tw, st)
  FFT_DISPATCH(g.log2nx, SPX_ROWS)
#undef SPX_ROWS
}

template <bool INV>
static void launch_cols(const Grid& g, const ColArgs& a, int nf, const float2* tw, cudaStream_t st,
                        const ColArgs* tab = nullptr, int nm = 1) {
#define SPX_COLS(L) launch_cols_n<INV, L>(g, a, tab, nf, nm, tw, st)
  FFT_DISPATCH(g.log2ny, SPX_COLS)
#undef SPX_COLS
}

// The half-spectrum arrays as a grid of nx/2 columns (the column transforms'
// view; the spatial pitch W is not used there).
static Grid half_grid(const Grid& g) {
  Grid h = g;
  h.nx = g.nx / 2;
  h.log2nx = g.log2nx - 1;
  return h;
}

void FieldBuffers::allocate(const Grid& grid) {
  g = grid;
  const size_t ss = g.spatial_size() * sizeof(float);
  for (int i = 0; i < SPX_NUM_FIELDS; ++i) {
    SPX_CUDA_TRY(cudaMalloc(&spatial[i], ss));
    SPX_CUDA_TRY(cudaMemset(spatial[i], 0, ss));
  }
  for (int i = 0; i < 4; ++i) {
    SPX_CUDA_TRY(cudaMalloc(&filt_tmp[i], ss));
    SPX_CUDA_TRY(cudaMemset(filt_tmp[i], 0, ss));
  }
  const size_t cs = g.half_spectral_size() * sizeof(float2);
  for (int i = 0; i < SP_COUNT; ++i) {
    SPX_CUDA_TRY(cudaMalloc(&spec[i], cs));
    SPX_CUDA_TRY(cudaMemset(spec[i], 0, cs));
  }
  for (auto [dst, n] : {std::pair<float2**, int>{&tw_x, g.nx}, {&tw_y, g.ny}}) {
    const std::vector<float2> t = make_pass_twiddles(n);
    SPX_CUDA_TRY(cudaMalloc(dst, t.size() * sizeof(float2)));
    SPX_CUDA_TRY(cudaMemcpy(*dst, t.data(), t.size() * sizeof(float2), cudaMemcpyHostToDevice));
  }
}

void FieldBuffers::release() {
  for (auto& p : spatial) { if (p) cudaFree(p); p = nullptr; }
  for (auto& p : filt_tmp) { if (p) cudaFree(p); p = nullptr; }
  for (auto& p : spec) { if (p) cudaFree(p); p = nullptr; }
  if (tw_x) cudaFree(tw_x);
  if (tw_y) cudaFree(tw_y);
  tw_x = tw_y = nullptr;
}

// The arguments of Flds::update's kernels for one simulation (shared by its own
// field_update and by a batch's tables, so both launch the same work).
static void source_lists(const FieldBuffers& fb, FieldList& zero, ConstFieldList& fsrc, FieldList& fdst) {
  zero = FieldList{};
  fsrc = ConstFieldList{};
  fdst = FieldList{};
  const int ids[5] = {SPX_JX, SPX_JY, SPX_JZ, SPX_DSTY, SPX_DENS};
  for (int i = 0; i < 5; ++i) zero.f[i] = fb.spatial[ids[i]];
  for (int i = 0; i < 4; ++i) {
    fsrc.f[i] = fb.spatial[ids[i]];
    fdst.f[i] = fb.filt_tmp[i];
  }
}
// copy_to_spectral (+ dsty/dens) fused with the row FFTs (mod.rs:66-85, 101-103, 122-124);
// fused: the sources come filtered from filt_tmp and are stored back into the fields
// with their periodic ghosts, the state the reference leaves.
static RowArgs rows_fwd_args(const FieldBuffers& fb, bool fused) {
  RowArgs a{};
  const int src_ids[7] = {SPX_JX, SPX_JY, SPX_JZ, SPX_DSTY, SPX_EX, SPX_EY, SPX_EZ};
  const int dst_ids[7] = {SP_JX, SP_JY, SP_JZ, SP_RHO, SP_EX, SP_EY, SP_EZ};
  for (int i = 0; i < 7; ++i) {
    a.src[i] = fb.spatial[src_ids[i]];
    a.dst[i] = fb.spec[dst_ids[i]];
    a.back[i] = nullptr;
    a.scale[i] = 1.0f;
  }
  if (fused)
    for (int i = 0; i < 4; ++i) {
      a.src[i] = fb.filt_tmp[i];
      a.back[i] = fb.spatial[src_ids[i]];
    }
  a.scale[3] = 1.0f / (float)fb.dens;
  return a;
}
static ColArgs cols_fwd_args(const FieldBuffers& fb) {
  const int dst_ids[7] = {SP_JX, SP_JY, SP_JZ, SP_RHO, SP_EX, SP_EY, SP_EZ};
  ColArgs c{};
  for (int i = 0; i < 7; ++i) c.data[i] = fb.spec[dst_ids[i]];
  return c;
}
static KArgs kspace_args(const FieldBuffers& fb) {
  KArgs k;
  k.jx = fb.spec[SP_JX]; k.jy = fb.spec[SP_JY]; k.jz = fb.spec[SP_JZ]; k.rho = fb.spec[SP_RHO];
  k.ex = fb.spec[SP_EX]; k.ey = fb.spec[SP_EY]; k.ez = fb.spec[SP_EZ];
  k.bwx = fb.spec[SP_BWX]; k.bwy = fb.spec[SP_BWY]; k.bwz = fb.spec[SP_BWZ];
  k.bax = fb.spec[SP_BAX]; k.bay = fb.spec[SP_BAY]; k.baz = fb.spec[SP_BAZ];
  k.ckc = fb.dt / (float)fb.dens;  // mod.rs:127
  k.cdt = fb.dt * fb.c;            // mod.rs:128
  return k;
}
// inverse transforms of B(t) and E, back to the spatial fields (mod.rs:281-307)
static const int kInvSpec[6] = {SP_BAX, SP_BAY, SP_BAZ, SP_EX, SP_EY, SP_EZ};
static ColArgs cols_inv_args(const FieldBuffers& fb) {
  ColArgs c{};
  for (int i = 0; i < 6; ++i) c.data[i] = fb.spec[kInvSpec[i]];
  return c;
}
static RowArgs rows_inv_args(const FieldBuffers& fb) {
  const int sp_ids[6] = {SPX_BX, SPX_BY, SPX_BZ, SPX_EX, SPX_EY, SPX_EZ};
  RowArgs a{};
  const float norm = 1.0f / (float)((uint64_t)fb.g.nx * (uint64_t)fb.g.ny);  // fft_2d.rs:170
  for (int i = 0; i < 6; ++i) {
    a.src[i] = fb.spec[kInvSpec[i]];
    a.dst[i] = fb.spatial[sp_ids[i]];
    a.scale[i] = norm;
  }
  return a;
}
static int kspace_blocks(const Grid& g, int nm) {
  const size_t n = g.half_spectral_size();
  return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)148 * 16 / (size_t)nm));
}

int field_update(FieldBuffers& fb, cudaStream_t st) {
  const Grid& g = fb.g;
  int launches = 0;
  // 1. n_pass binomial passes on jx, jy, jz, dsty (mod.rs:90-94).  Fused: all
  // passes in one kernel into filt_tmp.
  float* srcs[4] = {fb.spatial[SPX_JX], fb.spatial[SPX_JY], fb.spatial[SPX_JZ], fb.spatial[SPX_DSTY]};
  const bool fused = filter_fused_fits(fb.n_pass);
  if (fused) {
    launch_filter_fused(g, srcs, fb.filt_tmp, 4, fb.n_pass, st);
    ++launches;
  } else {  // separate passes, ping-pong (no filter when n_pass == 0)
    float* cur[4] = {srcs[0], srcs[1], srcs[2], srcs[3]};
    float* oth[4] = {fb.filt_tmp[0], fb.filt_tmp[1], fb.filt_tmp[2], fb.filt_tmp[3]};
    for (uint32_t p = 0; p < fb.n_pass; ++p) {
      launch_filter_pass(g, cur, oth, 4, st);
      ++launches;
      for (int i = 0; i < 4; ++i) std::swap(cur[i], oth[i]);
    }
    if (fb.n_pass & 1) {  // keep the filtered result in the field's own buffer
      for (int i = 0; i < 4; ++i)
        SPX_CUDA_TRY(cudaMemcpyAsync(oth[i], cur[i], g.spatial_size() * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
  }
  // 2. forward transforms
  launch_pair_rows<false>(g, rows_fwd_args(fb, fused), 7, fb.tw_x, st);
  launch_cols<false>(half_grid(g), cols_fwd_args(fb), 7, fb.tw_y, st);
  launches += 2;
  // 3. k-space update (mod.rs:105-278)
  k_kspace<<<kspace_blocks(g, 1), 256, 0, st>>>(kspace_args(fb), nullptr, g);
  ++launches;
  // 4. inverse transforms
  launch_cols<true>(half_grid(g), cols_inv_args(fb), 6, fb.tw_y, st);
  launch_pair_rows<true>(g, rows_inv_args(fb), 6, fb.tw_x, st);
  launches += 2;
  SPX_CUDA_TRY(cudaGetLastError());
  return launches;
}

// ---------------------------------------------------------------- batches
// The field phase of many simulations.  Members with the same grid and filter
// pass count form a group; each kernel of the phase (source zeroing, ghost fold,
// fused filter, the four transforms, the k-space update) runs once per group over
// all its members (blockIdx.z, or blockIdx.y for k_kspace, picks the member),
// reading the member's buffers and constants from a device table built once.
// The kernels and their arithmetic are the single simulation's, so every member's
// fields are bit-identical to its own field_update.  Groups run concurrently on
// streams of their own.
__global__ void k_zero_fields(const FieldList* __restrict__ tab, size_t n4) {
  float4* f = reinterpret_cast<float4*>(tab[blockIdx.z].f[blockIdx.y]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n4; i += (size_t)gridDim.x * blockDim.x)
    f[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

struct FieldGroup {
  Grid g{};
  uint32_t n_pass = 0;
  std::vector<FieldBuffers*> fbs;
  void* dev = nullptr;  // one allocation for the tables below
  FieldList* zero = nullptr;       // jx, jy, jz, dsty, dens: zeroed and folded
  ConstFieldList* fsrc = nullptr;  // filter inputs
  FieldList* fdst = nullptr;       // filter outputs (filt_tmp)
  RowArgs* rf = nullptr;
  ColArgs* cf = nullptr;
  KArgs* ks = nullptr;
  ColArgs* ci = nullptr;
  RowArgs* ri = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
};
struct FieldBatch {
  std::vector<FieldGroup> groups;
  cudaEvent_t fork = nullptr;
};

void field_batch_release(FieldBatch* b) {
  if (!b) return;
  for (FieldGroup& G : b->groups) {
    if (G.st) cudaStreamSynchronize(G.st);
    if (G.dev) cudaFree(G.dev);
    if (G.done) cudaEventDestroy(G.done);
    if (G.st) cudaStreamDestroy(G.st);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
}

FieldBatch* field_batch_build(const std::vector<FieldBuffers*>& members) {
  FieldBatch* b = new FieldBatch();
  try {
    for (FieldBuffers* fb : members) {
      FieldGroup* G = nullptr;
      for (FieldGroup& h : b->groups)  // (a group's members * 4 filtered fields index gridDim.z <= 65535)
        if (h.g.nx == fb->g.nx && h.g.ny == fb->g.ny && h.n_pass == fb->n_pass && h.fbs.size() < 16383) G = &h;
      if (!G) {
        b->groups.emplace_back();
        G = &b->groups.back();
        G->g = fb->g;
        G->n_pass = fb->n_pass;
      }
      G->fbs.push_back(fb);
    }
    SPX_CUDA_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (FieldGroup& G : b->groups) {
      const size_t nm = G.fbs.size();
      auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
      const size_t sz[8] = {up(nm * sizeof(FieldList)), up(nm * sizeof(ConstFieldList)), up(nm * sizeof(FieldList)),
                            up(nm * sizeof(RowArgs)),   up(nm * sizeof(ColArgs)),        up(nm * sizeof(KArgs)),
                            up(nm * sizeof(ColArgs)),   up(nm * sizeof(RowArgs))};
      size_t total = 0;
      for (size_t v : sz) total += v;
      std::vector<unsigned char> host(total, 0);
      SPX_CUDA_TRY(cudaMalloc(&G.dev, total));
      unsigned char* d = static_cast<unsigned char*>(G.dev);
      size_t off[8];
      for (int k = 0, o = 0; k < 8; o += (int)sz[k], ++k) off[k] = (size_t)o;
      G.zero = reinterpret_cast<FieldList*>(d + off[0]);
      G.fsrc = reinterpret_cast<ConstFieldList*>(d + off[1]);
      G.fdst = reinterpret_cast<FieldList*>(d + off[2]);
      G.rf = reinterpret_cast<RowArgs*>(d + off[3]);
      G.cf = reinterpret_cast<ColArgs*>(d + off[4]);
      G.ks = reinterpret_cast<KArgs*>(d + off[5]);
      G.ci = reinterpret_cast<ColArgs*>(d + off[6]);
      G.ri = reinterpret_cast<RowArgs*>(d + off[7]);
      const bool fused = filter_fused_fits(G.n_pass);
      for (size_t m = 0; m < nm; ++m) {
        const FieldBuffers& fb = *G.fbs[m];
        FieldList z;
        ConstFieldList fs;
        FieldList fd;
        source_lists(fb, z, fs, fd);
        const RowArgs rf = rows_fwd_args(fb, fused), ri = rows_inv_args(fb);
        const ColArgs cf = cols_fwd_args(fb), ci = cols_inv_args(fb);
        const KArgs ks = kspace_args(fb);
        std::memcpy(&host[off[0] + m * sizeof(FieldList)], &z, sizeof z);
        std::memcpy(&host[off[1] + m * sizeof(ConstFieldList)], &fs, sizeof fs);
        std::memcpy(&host[off[2] + m * sizeof(FieldList)], &fd, sizeof fd);
        std::memcpy(&host[off[3] + m * sizeof(RowArgs)], &rf, sizeof rf);
        std::memcpy(&host[off[4] + m * sizeof(ColArgs)], &cf, sizeof cf);
        std::memcpy(&host[off[5] + m * sizeof(KArgs)], &ks, sizeof ks);
        std::memcpy(&host[off[6] + m * sizeof(ColArgs)], &ci, sizeof ci);
        std::memcpy(&host[off[7] + m * sizeof(RowArgs)], &ri, sizeof ri);
      }
      SPX_CUDA_TRY(cudaMemcpy(G.dev, host.data(), total, cudaMemcpyHostToDevice));
      SPX_CUDA_TRY(cudaStreamCreateWithFlags(&G.st, cudaStreamNonBlocking));
      SPX_CUDA_TRY(cudaEventCreateWithFlags(&G.done, cudaEventDisableTiming));
    }
  } catch (...) {
    field_batch_release(b);
    throw;
  }
  return b;
}

int field_batch_groups(const FieldBatch* b) { return b ? (int)b->groups.size() : 0; }

int field_batch_zero_sources(FieldBatch* b, cudaStream_t st) {
  int launches = 0;
  for (FieldGroup& G : b->groups) {
    const size_t n = G.g.spatial_size();
    const int nm = (int)G.fbs.size();
    if (n % 4 == 0) {
      const int bx = (int)std::max<size_t>(1, std::min<size_t>((n / 4 + 255) / 256, 64));
      k_zero_fields<<<dim3(bx, 5, nm), 256, 0, st>>>(G.zero, n / 4);
      ++launches;
    } else {  // odd ghosted sizes: per field
      for (FieldBuffers* fb : G.fbs)
        for (int f : {SPX_JX, SPX_JY, SPX_JZ, SPX_DSTY, SPX_DENS}) {
          SPX_CUDA_TRY(cudaMemsetAsync(fb->spatial[f], 0, n * sizeof(float), st));
          ++launches;
        }
    }
  }
  SPX_CUDA_TRY(cudaGetLastError());
  return launches;
}

int field_batch_update(FieldBatch* b, cudaStream_t st) {
  int launches = 0;
  SPX_CUDA_TRY(cudaEventRecord(b->fork, st));
  for (FieldGroup& G : b->groups) {
    cudaStream_t gs = G.st;
    SPX_CUDA_TRY(cudaStreamWaitEvent(gs, b->fork, 0));
    const Grid& g = G.g;
    const int nm = (int)G.fbs.size();
    // Field::deposit_ghosts of the five sources (src/flds/field.rs:260-373)
    {
      const int nper = 2 * g.nx + 2 * (g.ny - 2);
      k_fold<<<dim3((nper + 255) / 256, 5, nm), 256, 0, gs>>>(FieldList{}, G.zero, g);
      ++launches;
    }
    if (!filter_fused_fits(G.n_pass)) {  // more passes than the fused filter holds: member by member
      for (FieldBuffers* fb : G.fbs) launches += field_update(*fb, gs);
    } else {
      const FieldBuffers& f0 = *G.fbs[0];  // twiddle tables depend on the grid only
      {
        const size_t smem = filter_fused_smem_floats((int)G.n_pass) * sizeof(float);
        const int tw = FILT_EW - 2 * ((int)G.n_pass - 1);
        const dim3 grd((g.nx + tw - 1) / tw, (g.ny + FILT_TY - 1) / FILT_TY, 4 * nm);
        k_filter_fused<<<grd, 256, smem, gs>>>(ConstFieldList{}, FieldList{}, G.fsrc, G.fdst, 4, g, (int)G.n_pass);
      }
      launch_pair_rows<false>(g, RowArgs{}, 7, f0.tw_x, gs, G.rf, nm);
      launch_cols<false>(half_grid(g), ColArgs{}, 7, f0.tw_y, gs, G.cf, nm);
      k_kspace<<<dim3(kspace_blocks(g, nm), nm), 256, 0, gs>>>(KArgs{}, G.ks, g);
      launch_cols<true>(half_grid(g), ColArgs{}, 6, f0.tw_y, gs, G.ci, nm);
      launch_pair_rows<true>(g, RowArgs{}, 6, f0.tw_x, gs, G.ri, nm);
      launches += 6;
    }
    SPX_CUDA_TRY(cudaEventRecord(G.done, gs));
    SPX_CUDA_TRY(cudaStreamWaitEvent(st, G.done, 0));
  }
  SPX_CUDA_TRY(cudaGetLastError());
  return launches;
}

int fft2d_inplace(const Grid& g, float2* data, const float2* tw_x, const float2* tw_y, bool inverse,
                  cudaStream_t st) {
  RowArgs a{};
  a.src[0] = data;
  a.dst[0] = data;
  ColArgs c{};
  c.data[0] = data;
  if (!inverse) {
    a.scale[0] = 1.0f;
    launch_rows<false>(g, a, 1, tw_x, st);
    launch_cols<false>(g, c, 1, tw_y, st);
  } else {
    // reference order: rows then columns, then the 1/(nx ny) scale (fft_2d.rs:132-172)
    a.scale[0] = 1.0f;
    launch_rows<true>(g, a, 1, tw_x, st);
    launch_cols<true>(g, c, 1, tw_y, st);
    const size_t n = g.spectral_size();
    const float norm = 1.0f / (float)n;
    k_scale_c<<<(int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(data, n, norm);
  }
  SPX_CUDA_TRY(cudaGetLastError());
  return 2;
}

}  // namespace spx
