// Particle kernels of the B200 hot path: the fused Boris push + move + deposit
// over the cell-slot layout (src/prtls.rs:86-443 and src/lib.rs:266-489 of the
// reference), its overflow fallback, pack/unpack, the plain FP32 baseline path,
// kinetic-energy diagnostics and seeded device initialisation.
//
// This translation unit is compiled with -fmad=false: the reference's Rust never
// fuses a*b+c, so no contraction is allowed here either.  Division and sqrt are
// the IEEE round-to-nearest operations (no fast math).  With identical inputs
// the particle state (cell indices, offsets, momenta) is then bit-identical to
// the reference's FP32 arithmetic.
#include <algorithm>

#include "particles.cuh"

namespace spx {

// ---------------------------------------------------------------- per-particle maths
// Second-order (TSC) weights, src/lib.rs:339-347, left-to-right as in Rust.
__device__ __forceinline__ void tsc_weights(float dx, float dy, float (&w)[9]) {
  w[0] = 0.5f * (0.5f - dy) * (0.5f - dy) * 0.5f * (0.5f - dx) * (0.5f - dx);
  w[1] = 0.5f * (0.5f - dy) * (0.5f - dy) * (0.75f - dx * dx);
  w[2] = 0.5f * (0.5f - dy) * (0.5f - dy) * 0.5f * (0.5f + dx) * (0.5f + dx);
  w[3] = (0.75f - dy * dy) * 0.5f * (0.5f - dx) * (0.5f - dx);
  w[4] = (0.75f - dy * dy) * (0.75f - dx * dx);
  w[5] = (0.75f - dy * dy) * 0.5f * (0.5f + dx) * (0.5f + dx);
  w[6] = 0.5f * (0.5f + dy) * (0.5f + dy) * 0.5f * (0.5f - dx) * (0.5f - dx);
  w[7] = 0.5f * (0.5f + dy) * (0.5f + dy) * (0.75f - dx * dx);
  w[8] = 0.5f * (0.5f + dy) * (0.5f + dy) * 0.5f * (0.5f + dx) * (0.5f + dx);
}

// Boris push of src/prtls.rs:412-440 given the gathered fields g[0..5] = E, B.
__device__ __forceinline__ void boris(const float (&g)[6], float beta, float alpha, float csqinv, float& px,
                                      float& py, float& pz, float& psa) {
  const float ext = g[0] * beta, eyt = g[1] * beta, ezt = g[2] * beta;
  float bxt = g[3] * alpha, byt = g[4] * alpha, bzt = g[5] * alpha;
  const float ux = px + ext, uy = py + eyt, uz = pz + ezt;
  const float gt = 1.0f / sqrtf(1.0f + (ux * ux + uy * uy + uz * uz) * csqinv);
  bxt *= gt;
  byt *= gt;
  bzt *= gt;
  const float boris = 2.0f * (1.0f / (1.0f + bxt * bxt + byt * byt + bzt * bzt));
  const float uxt = ux + uy * bzt - uz * byt;
  const float uyt = uy + uz * bxt - ux * bzt;
  const float uzt = uz + ux * byt - uy * bxt;
  px = ux + boris * (uyt * bzt - uzt * byt) + ext;
  py = uy + boris * (uzt * bxt - uxt * bzt) + eyt;
  pz = uz + boris * (uxt * byt - uyt * bxt) + ezt;
  psa = sqrtf(1.0f + (px * px + py * py + pz * pz) * csqinv);
}

__device__ __forceinline__ float gamma_of(float px, float py, float pz, float csqinv) {
  return sqrtf(1.0f + (px * px + py * py + pz * pz) * csqinv);  // src/prtls.rs:440
}

// update_position (src/prtls.rs:103-119) for one particle; inv = 1/psa.
__device__ __forceinline__ void move_half(float c1, float px, float py, int& ix, int& iy, float& dx, float& dy) {
  dx += c1 * px;
  if (dx >= 0.5f) {
    dx -= 1.0f;
    ix += 1;
  } else if (dx < -0.5f) {
    dx += 1.0f;
    ix -= 1;
  }
  dy += c1 * py;
  if (dy >= 0.5f) {
    dy -= 1.0f;
    iy += 1;
  } else if (dy < -0.5f) {
    dy += 1.0f;
    iy -= 1;
  }
}

// apply_bc (src/prtls.rs:124-190) for one particle.  The reference asserts
// max(ix) <= wall_loc + 1 and min(ix) > delta over the species before the wall
// pass; here each particle checks itself and raises the device error word.
__device__ __forceinline__ void apply_bc(const PhysParams& p, int nx, int ny, int& ix, int& iy, float& dx, float& px,
                                         int* derr) {
  if (iy < 1)
    iy += ny;
  else if (iy > ny)
    iy -= ny;
  if (p.periodic_x) {
    if (ix < 1)
      ix += nx;
    else if (ix > nx)
      ix -= nx;
  } else {
    if (ix > p.wall_loc + 1 || ix < p.delta + (p.left_wall ? 0 : 1)) atomicOr(derr, DERR_WALL);
    if (p.left_wall && ix <= p.delta + 1) {  // optional mirror image of the right wall
      if (ix == p.delta + 1) {
        const float sgn = isnan(dx) ? dx : copysignf(1.0f, dx);
        if (sgn < 0.0f) {
          px *= -1.0f;
          dx *= -1.0f;
        }
      } else {
        dx -= 1.0f;
        ix += 1;
        px *= -1.0f;
      }
      return;
    }
    if (ix < p.wall_loc) {
    } else if (ix == p.wall_loc) {
      const float sgn = isnan(dx) ? dx : copysignf(1.0f, dx);  // f32::signum
      px *= -sgn;
      dx *= -sgn;
    } else {
      dx += 1.0f;
      ix -= 1;
      px *= -1.0f;
    }
  }
}

// ---------------------------------------------------------------- split path kernel
struct SpeciesArgs {
  // read buffer
  const float *dx, *dy, *px, *py, *pz;
  const uint32_t* tag;
  const uint32_t *nlow, *ntop;
  float *rpx, *rpy, *rpz;  // in-place momentum writes (push-only mode)
  // write buffer
  float *wdx, *wdy, *wpx, *wpy, *wpz;
  uint32_t* wtag;
  uint32_t *wnlow, *wntop;
  // overflow lists: read (r*) and write (w*)
  const uint32_t* rocell;
  const float *rodx, *rody, *ropx, *ropy, *ropz;
  const uint32_t* rotag;
  float *ropx_w, *ropy_w, *ropz_w;
  uint32_t* wocell;
  float *wodx, *wody, *wopx, *wopy, *wopz;
  uint32_t* wotag;
  const uint32_t* rocount;
  uint32_t* wocount;
  uint32_t ocap;
  float charge, alpha, beta;
  int K;
};

struct StepArgs {
  SpeciesArgs sp[MAX_SPECIES];
  int ns;
  FieldPtrs f;
  Grid g;
  int TX, TY, logTX, logTY, NTX;
  PhysParams p;
  int* derr;
};

// Deposit v * w[k] on the 3x3 stencil centred on (ix, iy): into the CTA's
// shared window when it fits, otherwise straight into the global field.
__device__ __forceinline__ void dep9(float* win, int WX, int WY, int wx0, int wy0, float* glob, int W, int ix, int iy,
                                     const float (&w)[9], float v) {
  const int lx = ix - wx0, ly = iy - wy0;
  if (lx >= 1 && lx <= WX - 2 && ly >= 1 && ly <= WY - 2) {
    float* b = win + (ly - 1) * WX + (lx - 1);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q) atomicAdd(b + r * WX + q, w[r * 3 + q] * v);
  } else {
    float* b = glob + (size_t)(iy - 1) * W + (ix - 1);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q) atomicAdd(b + (size_t)r * W + q, w[r * 3 + q] * v);
  }
}

// Append a particle that left its cell to the destination cell's top slots of
// the write buffer (or to the overflow list).
__device__ __forceinline__ void relocate(const StepArgs& a, const SpeciesArgs& S, int ix, int iy, float dx, float dy,
                                         float px, float py, float pz, uint32_t tag) {
  const int TC = a.TX * a.TY;
  const int dtx = (ix - 1) >> a.logTX, dty = (iy - 1) >> a.logTY;
  const int dc = (((iy - 1) & (a.TY - 1)) << a.logTX) | ((ix - 1) & (a.TX - 1));
  const size_t dtile = (size_t)dty * a.NTX + dtx;
  const size_t dgc = dtile * TC + dc;
  const int limit = S.K - (int)(S.nlow[dgc] + S.ntop[dgc]);
  const int i = (int)atomicAdd(&S.wntop[dgc], 1u);
  if (i < limit) {
    const size_t widx = dtile * (size_t)S.K * TC + (size_t)(S.K - 1 - i) * TC + dc;
    S.wdx[widx] = dx;
    S.wdy[widx] = dy;
    S.wpx[widx] = px;
    S.wpy[widx] = py;
    S.wpz[widx] = pz;
    S.wtag[widx] = tag;
  } else {
    atomicSub(&S.wntop[dgc], 1u);
    const uint32_t o = atomicAdd(S.wocount, 1u);
    if (o < S.ocap) {
      S.wocell[o] = (uint32_t)ix | ((uint32_t)iy << 16);
      S.wodx[o] = dx;
      S.wody[o] = dy;
      S.wopx[o] = px;
      S.wopy[o] = py;
      S.wopz[o] = pz;
      S.wotag[o] = tag;
    } else {
      atomicOr(a.derr, DERR_OVERFLOW_LOST);
    }
  }
}

// Shared-memory pitch of the E/B window: the lanes of a warp cover 32/TX tile
// rows; a pitch congruent to TX modulo 32 puts consecutive rows on disjoint
// banks, so every gather load of a warp is conflict-free.
__host__ __device__ inline int eb_pitch(int TX) {
  if (TX >= 32) return TX + 2;
  int p = TX;
  while (p < TX + 2) p += 32;
  return p;
}

// One CTA per tile, one thread per cell.  Every particle a thread processes
// starts in the thread's cell: the E/B window of the tile (+1 cell halo) is
// staged once in shared memory and gathered with conflict-free loads, and
// deposits that stay in the cell's 3x3 stencil accumulate in registers (36
// accumulators); only particles whose half- or full-step cell differs use
// shared-memory atomics.  The next particle's state is loaded while the
// current one is processed.
template <bool PUSH, bool MOVE>
__global__ void __launch_bounds__(256, 2) k_slot(const __grid_constant__ StepArgs a) {
  extern __shared__ float smem[];
  const int TC = a.TX * a.TY;
  const int tile = blockIdx.x;
  const int tx = tile % a.NTX, ty = tile / a.NTX;
  const int c = threadIdx.x;
  const int lx = c & (a.TX - 1), ly = c >> a.logTX;
  const int ox = tx * a.TX + lx + 1, oy = ty * a.TY + ly + 1;  // owner cell (reference coords)
  const int W = a.g.W, nx = a.g.nx, ny = a.g.ny;
  // deposit window: tile + 2 cells
  const int WX = a.TX + 4, WY = a.TY + 4, WN = WX * WY;
  const int wx0 = tx * a.TX + 1 - 2, wy0 = ty * a.TY + 1 - 2;
  float* win = smem;
  float* wjx = win;
  float* wjy = win + WN;
  float* wjz = win + 2 * WN;
  float* wrho = win + 3 * WN;
  float* wdens = win + 4 * WN;
  // E/B window: tile + 1 cell, 6 planes
  const int PE = eb_pitch(a.TX), EY = a.TY + 2, EN = PE * EY;
  float* ebw = smem + (MOVE ? 5 * WN : 0);
  if (MOVE)
    for (int i = c; i < 5 * WN; i += TC) win[i] = 0.f;
  if (PUSH) {
    const float* src[6] = {a.f.E[0], a.f.E[1], a.f.E[2], a.f.B[0], a.f.B[1], a.f.B[2]};
    const int EX = a.TX + 2;
    for (int i = c; i < 6 * EY * EX; i += TC) {
      const int f = i / (EY * EX), k = i - f * (EY * EX);
      const int r = k / EX, q = k - r * EX;
      ebw[f * EN + r * PE + q] = __ldg(src[f] + (size_t)(ty * a.TY + r) * W + (tx * a.TX + q));
    }
  }
  __syncthreads();
  const float* eb = ebw + ly * PE + lx;  // top-left of this cell's 3x3 neighbourhood
  float accJ[3][9];
#pragma unroll
  for (int k = 0; k < 9; ++k) accJ[0][k] = accJ[1][k] = accJ[2][k] = 0.f;
  const size_t gc = (size_t)tile * TC + c;
  const float half_dt = 0.5f * a.p.dt;
  const float csqinv = a.p.csqinv;

  for (int s = 0; s < a.ns; ++s) {
    const SpeciesArgs& S = a.sp[s];
    const float* __restrict__ rdx = S.dx;
    const float* __restrict__ rdy = S.dy;
    const float* __restrict__ rpx = S.px;
    const float* __restrict__ rpy = S.py;
    const float* __restrict__ rpz = S.pz;
    const uint32_t* __restrict__ rtag = S.tag;
    const int K = S.K;
    const size_t base = (size_t)tile * K * TC + c;
    const int nlow = (int)S.nlow[gc], ntop = (int)S.ntop[gc];
    const int total = nlow + ntop;
    const float q = S.charge, beta = S.beta, alpha = S.alpha;
    float accD[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) accD[k] = 0.f;
    int wcur = 0;
    // software pipeline: state of particle n is loaded during particle n-1
    float ndx = 0.f, ndy = 0.f, npx = 0.f, npy = 0.f, npz = 0.f;
    uint32_t ntag = 0;
    size_t nidx = base;
    if (total > 0) {
      nidx = base + (size_t)(nlow > 0 ? 0 : K - 1) * TC;
      ndx = rdx[nidx];
      ndy = rdy[nidx];
      npx = rpx[nidx];
      npy = rpy[nidx];
      npz = rpz[nidx];
      if (MOVE) ntag = rtag[nidx];
    }
    for (int n = 0; n < total; ++n) {
      const size_t idx = nidx;
      float dx = ndx, dy = ndy, px = npx, py = npy, pz = npz;
      const uint32_t tag = ntag;
      if (n + 1 < total) {
        const int m = n + 1;
        const int slot = m < nlow ? m : K - 1 - (m - nlow);
        nidx = base + (size_t)slot * TC;
        ndx = rdx[nidx];
        ndy = rdy[nidx];
        npx = rpx[nidx];
        npy = rpy[nidx];
        npz = rpz[nidx];
        if (MOVE) ntag = rtag[nidx];
      }
      float psa;
      if (PUSH) {
        float w[9];
        tsc_weights(dx, dy, w);
        float gth[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) {
          const float* e = eb + f * EN;
          float t = w[0] * e[0];
          t += w[1] * e[1];
          t += w[2] * e[2];
          t += w[3] * e[PE];
          t += w[4] * e[PE + 1];
          t += w[5] * e[PE + 2];
          t += w[6] * e[2 * PE];
          t += w[7] * e[2 * PE + 1];
          t += w[8] * e[2 * PE + 2];
          gth[f] = t;
        }
        boris(gth, beta, alpha, csqinv, px, py, pz, psa);
      } else {
        psa = gamma_of(px, py, pz, csqinv);
      }
      if (!MOVE) {
        S.rpx[idx] = px;
        S.rpy[idx] = py;
        S.rpz[idx] = pz;
        continue;
      }
      const float inv = 1.0f / psa;
      const float c1 = half_dt * inv;
      int ix = ox, iy = oy;
      // first half: position, boundaries, current (src/lib.rs:480-484)
      move_half(c1, px, py, ix, iy, dx, dy);
      apply_bc(a.p, nx, ny, ix, iy, dx, px, a.derr);
      {
        const float vx = q * px * inv, vy = q * py * inv, vz = q * pz * inv;
        float w[9];
        tsc_weights(dx, dy, w);
        if (ix == ox && iy == oy) {
#pragma unroll
          for (int k = 0; k < 9; ++k) {
            accJ[0][k] += w[k] * vx;
            accJ[1][k] += w[k] * vy;
            accJ[2][k] += w[k] * vz;
          }
        } else {
          dep9(wjx, WX, WY, wx0, wy0, a.f.J[0], W, ix, iy, w, vx);
          dep9(wjy, WX, WY, wx0, wy0, a.f.J[1], W, ix, iy, w, vy);
          dep9(wjz, WX, WY, wx0, wy0, a.f.J[2], W, ix, iy, w, vz);
        }
      }
      // second half: position, boundaries, density (src/lib.rs:486-488)
      move_half(c1, px, py, ix, iy, dx, dy);
      apply_bc(a.p, nx, ny, ix, iy, dx, px, a.derr);
      {
        float w[9];
        tsc_weights(dx, dy, w);
        if (ix == ox && iy == oy) {
#pragma unroll
          for (int k = 0; k < 9; ++k) accD[k] += w[k];
        } else {
          dep9(wrho, WX, WY, wx0, wy0, a.f.dsty, W, ix, iy, w, q);
          dep9(wdens, WX, WY, wx0, wy0, a.f.dens, W, ix, iy, w, 1.0f);
        }
      }
      if (ix == ox && iy == oy) {
        const size_t widx = base + (size_t)wcur * TC;
        S.wdx[widx] = dx;
        S.wdy[widx] = dy;
        S.wpx[widx] = px;
        S.wpy[widx] = py;
        S.wpz[widx] = pz;
        S.wtag[widx] = tag;
        ++wcur;
      } else {
        relocate(a, S, ix, iy, dx, dy, px, py, pz, tag);
      }
    }
    if (MOVE) {
      S.wnlow[gc] = (uint32_t)wcur;
      // this species' density stencil of the owner cell -> window
      const int bl = (oy - 1 - wy0) * WX + (ox - 1 - wx0);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float d = accD[r * 3 + k];
          if (d != 0.f) {
            atomicAdd(wrho + bl + r * WX + k, d * q);
            atomicAdd(wdens + bl + r * WX + k, d);
          }
        }
    }
  }
  if (!MOVE) return;
  {
    const int bl = (oy - 1 - wy0) * WX + (ox - 1 - wx0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        atomicAdd(wjx + bl + r * WX + k, accJ[0][r * 3 + k]);
        atomicAdd(wjy + bl + r * WX + k, accJ[1][r * 3 + k]);
        atomicAdd(wjz + bl + r * WX + k, accJ[2][r * 3 + k]);
      }
  }
  __syncthreads();
  // window -> global (clipped to the ghosted grid)
  float* dst[5] = {a.f.J[0], a.f.J[1], a.f.J[2], a.f.dsty, a.f.dens};
  for (int i = c; i < 5 * WN; i += TC) {
    const float v = win[i];
    if (v == 0.f) continue;
    const int plane = i / WN, k = i - plane * WN;
    const int wy = k / WX, wx = k - wy * WX;
    const int gx = wx0 + wx, gy = wy0 + wy;
    if (gx < 0 || gx > nx + 1 || gy < 0 || gy > ny + 1) continue;
    atomicAdd(dst[plane] + (size_t)gy * W + gx, v);
  }
}

// Overflow fallback: particles parked in the overflow list (no free slot in
// their cell) get the same per-particle work with global gathers and global
// atomic deposits.
template <bool PUSH, bool MOVE>
__global__ void k_slot_overflow(const __grid_constant__ StepArgs a, int s) {
  const SpeciesArgs& S = a.sp[s];
  const uint32_t n = min(*S.rocount, S.ocap);
  const int W = a.g.W, nx = a.g.nx, ny = a.g.ny;
  const float csqinv = a.p.csqinv;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t cell = S.rocell[i];
    int ix = (int)(cell & 0xFFFFu), iy = (int)(cell >> 16);
    float dx = S.rodx[i], dy = S.rody[i], px = S.ropx[i], py = S.ropy[i], pz = S.ropz[i];
    float psa;
    if (PUSH) {
      float w[9];
      tsc_weights(dx, dy, w);
      const float* src[6] = {a.f.E[0], a.f.E[1], a.f.E[2], a.f.B[0], a.f.B[1], a.f.B[2]};
      float gth[6];
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const float* b = src[f] + (size_t)(iy - 1) * W + (ix - 1);
        float t = w[0] * b[0];
        t += w[1] * b[1];
        t += w[2] * b[2];
        t += w[3] * b[W];
        t += w[4] * b[W + 1];
        t += w[5] * b[W + 2];
        t += w[6] * b[2 * W];
        t += w[7] * b[2 * W + 1];
        t += w[8] * b[2 * W + 2];
        gth[f] = t;
      }
      boris(gth, S.beta, S.alpha, csqinv, px, py, pz, psa);
    } else {
      psa = gamma_of(px, py, pz, csqinv);
    }
    if (!MOVE) {
      S.ropx_w[i] = px;
      S.ropy_w[i] = py;
      S.ropz_w[i] = pz;
      continue;
    }
    const float q = S.charge;
    const float inv = 1.0f / psa;
    const float c1 = 0.5f * a.p.dt * inv;
    move_half(c1, px, py, ix, iy, dx, dy);
    apply_bc(a.p, nx, ny, ix, iy, dx, px, a.derr);
    {
      const float vx = q * px * inv, vy = q * py * inv, vz = q * pz * inv;
      float w[9];
      tsc_weights(dx, dy, w);
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
          const size_t o = (size_t)(iy - 1 + r) * W + (ix - 1 + k);
          atomicAdd(a.f.J[0] + o, w[r * 3 + k] * vx);
          atomicAdd(a.f.J[1] + o, w[r * 3 + k] * vy);
          atomicAdd(a.f.J[2] + o, w[r * 3 + k] * vz);
        }
    }
    move_half(c1, px, py, ix, iy, dx, dy);
    apply_bc(a.p, nx, ny, ix, iy, dx, px, a.derr);
    {
      float w[9];
      tsc_weights(dx, dy, w);
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) {
          const size_t o = (size_t)(iy - 1 + r) * W + (ix - 1 + k);
          atomicAdd(a.f.dsty + o, w[r * 3 + k] * q);
          atomicAdd(a.f.dens + o, w[r * 3 + k]);
        }
    }
    relocate(a, S, ix, iy, dx, dy, px, py, pz, S.rotag[i]);
  }
}

static SpeciesArgs species_args(Species& sp) {
  SlotSpecies& s = sp.slot;
  const int r = s.cur, w = s.cur ^ 1;
  SpeciesArgs A;
  A.dx = s.dx[r];
  A.dy = s.dy[r];
  A.px = s.px[r];
  A.py = s.py[r];
  A.pz = s.pz[r];
  A.tag = s.tag[r];
  A.nlow = s.nlow[r];
  A.ntop = s.ntop[r];
  A.rpx = s.px[r];
  A.rpy = s.py[r];
  A.rpz = s.pz[r];
  A.wdx = s.dx[w];
  A.wdy = s.dy[w];
  A.wpx = s.px[w];
  A.wpy = s.py[w];
  A.wpz = s.pz[w];
  A.wtag = s.tag[w];
  A.wnlow = s.nlow[w];
  A.wntop = s.ntop[w];
  A.rocell = s.ocell[r];
  A.rodx = s.odx[r];
  A.rody = s.ody[r];
  A.ropx = s.opx[r];
  A.ropy = s.opy[r];
  A.ropz = s.opz[r];
  A.rotag = s.otag[r];
  A.ropx_w = s.opx[r];
  A.ropy_w = s.opy[r];
  A.ropz_w = s.opz[r];
  A.wocell = s.ocell[w];
  A.wodx = s.odx[w];
  A.wody = s.ody[w];
  A.wopx = s.opx[w];
  A.wopy = s.opy[w];
  A.wopz = s.opz[w];
  A.wotag = s.otag[w];
  A.rocount = s.ocount + r;
  A.wocount = s.ocount + w;
  A.ocap = s.ocap;
  A.charge = sp.charge;
  A.alpha = sp.alpha;
  A.beta = sp.beta;
  A.K = s.K;
  return A;
}

int slot_step(Species* sp, int s0, int s1, const ParticleGeom& pg, const PhysParams& pp, const FieldPtrs& fp,
              bool push, bool move, int* derr, cudaStream_t st) {
  StepArgs a;
  a.ns = s1 - s0;
  a.f = fp;
  a.g = pg.g;
  a.TX = pg.TX;
  a.TY = pg.TY;
  a.logTX = pg.logTX;
  a.logTY = pg.logTY;
  a.NTX = pg.NTX;
  a.p = pp;
  a.derr = derr;
  int launches = 0;
  for (int s = s0; s < s1; ++s) {
    a.sp[s - s0] = species_args(sp[s]);
    if (move) {
      SlotSpecies& S = sp[s].slot;
      const int w = S.cur ^ 1;
      SPX_CUDA_TRY(cudaMemsetAsync(S.ntop[w], 0, pg.ncells() * sizeof(uint32_t), st));
      SPX_CUDA_TRY(cudaMemsetAsync(S.ocount + w, 0, sizeof(uint32_t), st));
    }
  }
  const int TC = pg.TC();
  const size_t smem = ((move ? 5 * (size_t)(pg.TX + 4) * (pg.TY + 4) : 0) +
                       (push ? 6 * (size_t)eb_pitch(pg.TX) * (pg.TY + 2) : 0)) * sizeof(float);
  if (push && move)
    k_slot<true, true><<<pg.ntiles(), TC, smem, st>>>(a);
  else if (push)
    k_slot<true, false><<<pg.ntiles(), TC, smem, st>>>(a);
  else if (move)
    k_slot<false, true><<<pg.ntiles(), TC, smem, st>>>(a);
  ++launches;
  for (int s = 0; s < a.ns; ++s) {
    // the overflow fallback reads its count on the device; a small fixed grid covers it
    if (push && move)
      k_slot_overflow<true, true><<<64, 256, 0, st>>>(a, s);
    else if (push)
      k_slot_overflow<true, false><<<64, 256, 0, st>>>(a, s);
    else if (move)
      k_slot_overflow<false, true><<<64, 256, 0, st>>>(a, s);
    ++launches;
  }
  SPX_CUDA_TRY(cudaGetLastError());
  if (move)
    for (int s = s0; s < s1; ++s) sp[s].slot.cur ^= 1;
  return launches;
}

// ---------------------------------------------------------------- pack / unpack
__device__ __forceinline__ size_t cell_gc(uint32_t cell, int TX, int TY, int logTX, int logTY, int NTX) {
  const int ix = (int)(cell & 0xFFFFu), iy = (int)(cell >> 16);
  const int tx = (ix - 1) >> logTX, ty = (iy - 1) >> logTY;
  const int c = (((iy - 1) & (TY - 1)) << logTX) | ((ix - 1) & (TX - 1));
  return ((size_t)ty * NTX + tx) * (size_t)(TX * TY) + c;
}

__global__ void k_count(uint64_t n, const uint32_t* cell, uint32_t* counts, int TX, int TY, int logTX, int logTY,
                        int NTX) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(&counts[cell_gc(cell[i], TX, TY, logTX, logTY, NTX)], 1u);
}

__global__ void k_scatter(uint64_t n, const uint32_t* cell, const float* dx, const float* dy, const float* px,
                          const float* py, const float* pz, const uint32_t* tag, uint32_t* cursor, float* odx,
                          float* ody, float* opx, float* opy, float* opz, uint32_t* otag, int K, int TX, int TY,
                          int logTX, int logTY, int NTX) {
  const int TC = TX * TY;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const size_t gc = cell_gc(cell[i], TX, TY, logTX, logTY, NTX);
    const uint32_t r = atomicAdd(&cursor[gc], 1u);
    if ((int)r >= K) continue;  // cannot happen: K >= max count
    const size_t tile = gc / TC, c = gc - tile * TC;
    const size_t o = tile * (size_t)K * TC + (size_t)r * TC + c;
    odx[o] = dx[i];
    ody[o] = dy[i];
    opx[o] = px[i];
    opy[o] = py[i];
    opz[o] = pz[i];
    otag[o] = tag ? tag[i] : (uint32_t)i;
  }
}

void slot_count(const ParticleGeom& pg, uint64_t n, const uint32_t* cell, uint32_t* counts, cudaStream_t st) {
  SPX_CUDA_TRY(cudaMemsetAsync(counts, 0, pg.ncells() * sizeof(uint32_t), st));
  if (n) k_count<<<148 * 8, 256, 0, st>>>(n, cell, counts, pg.TX, pg.TY, pg.logTX, pg.logTY, pg.NTX);
  SPX_CUDA_TRY(cudaGetLastError());
}

void slot_scatter(Species& s, const ParticleGeom& pg, uint64_t n, const uint32_t* cell, const float* dx,
                  const float* dy, const float* px, const float* py, const float* pz, const uint32_t* tag,
                  uint32_t* cursor, cudaStream_t st) {
  SlotSpecies& S = s.slot;
  S.cur = 0;
  SPX_CUDA_TRY(cudaMemsetAsync(cursor, 0, pg.ncells() * sizeof(uint32_t), st));
  if (n)
    k_scatter<<<148 * 8, 256, 0, st>>>(n, cell, dx, dy, px, py, pz, tag, cursor, S.dx[0], S.dy[0], S.px[0], S.py[0],
                                       S.pz[0], S.tag[0], S.K, pg.TX, pg.TY, pg.logTX, pg.logTY, pg.NTX);
  SPX_CUDA_TRY(cudaMemcpyAsync(S.nlow[0], cursor, pg.ncells() * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  SPX_CUDA_TRY(cudaMemsetAsync(S.ntop[0], 0, pg.ncells() * sizeof(uint32_t), st));
  SPX_CUDA_TRY(cudaMemsetAsync(S.ocount, 0, 2 * sizeof(uint32_t), st));
  SPX_CUDA_TRY(cudaGetLastError());
}

__global__ void k_unpack(SpeciesArgs S, int TX, int TY, int logTX, int NTX, size_t ncells, uint32_t* ix,
                         uint32_t* iy, float* dx, float* dy, float* px, float* py, float* pz, float* psa,
                         float csqinv) {
  const int TC = TX * TY;
  for (size_t gc = blockIdx.x * (size_t)blockDim.x + threadIdx.x; gc < ncells; gc += (size_t)gridDim.x * blockDim.x) {
    const size_t tile = gc / TC;
    const int c = (int)(gc - tile * TC);
    const int tx = (int)(tile % NTX), ty = (int)(tile / NTX);
    const uint32_t cx = tx * TX + (c & (TX - 1)) + 1, cy = ty * TY + (c >> logTX) + 1;
    const int nlow = (int)S.nlow[gc], ntop = (int)S.ntop[gc];
    const size_t base = tile * (size_t)S.K * TC + c;
    for (int n = 0; n < nlow + ntop; ++n) {
      const int slot = n < nlow ? n : S.K - 1 - (n - nlow);
      const size_t i = base + (size_t)slot * TC;
      const uint32_t t = S.tag[i];
      if (ix) ix[t] = cx;
      if (iy) iy[t] = cy;
      if (dx) dx[t] = S.dx[i];
      if (dy) dy[t] = S.dy[i];
      if (px) px[t] = S.px[i];
      if (py) py[t] = S.py[i];
      if (pz) pz[t] = S.pz[i];
      if (psa) psa[t] = gamma_of(S.px[i], S.py[i], S.pz[i], csqinv);
    }
  }
}

__global__ void k_unpack_overflow(SpeciesArgs S, uint32_t* ix, uint32_t* iy, float* dx, float* dy, float* px,
                                  float* py, float* pz, float* psa, float csqinv) {
  const uint32_t n = min(*S.rocount, S.ocap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t t = S.rotag[i];
    const uint32_t cell = S.rocell[i];
    if (ix) ix[t] = cell & 0xFFFFu;
    if (iy) iy[t] = cell >> 16;
    if (dx) dx[t] = S.rodx[i];
    if (dy) dy[t] = S.rody[i];
    if (px) px[t] = S.ropx[i];
    if (py) py[t] = S.ropy[i];
    if (pz) pz[t] = S.ropz[i];
    if (psa) psa[t] = gamma_of(S.ropx[i], S.ropy[i], S.ropz[i], csqinv);
  }
}

void slot_unpack(const Species& s, const ParticleGeom& pg, uint32_t* ix, uint32_t* iy, float* dx, float* dy,
                 float* px, float* py, float* pz, float* psa, float csqinv, cudaStream_t st) {
  SpeciesArgs A = species_args(const_cast<Species&>(s));
  k_unpack<<<148 * 8, 256, 0, st>>>(A, pg.TX, pg.TY, pg.logTX, pg.NTX, pg.ncells(), ix, iy, dx, dy, px, py, pz, psa,
                                   csqinv);
  k_unpack_overflow<<<64, 256, 0, st>>>(A, ix, iy, dx, dy, px, py, pz, psa, csqinv);
  SPX_CUDA_TRY(cudaGetLastError());
}

__global__ void k_max_occ(const uint32_t* nlow, const uint32_t* ntop, size_t n, uint32_t* out) {
  uint32_t m = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = max(m, nlow[i] + ntop[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

void slot_max_occupancy(const Species& s, const ParticleGeom& pg, uint32_t* d_out, cudaStream_t st) {
  const SlotSpecies& S = s.slot;
  k_max_occ<<<148 * 4, 256, 0, st>>>(S.nlow[S.cur], S.ntop[S.cur], pg.ncells(), d_out);
  SPX_CUDA_TRY(cudaGetLastError());
}

void slot_allocate(Species& s, const ParticleGeom& pg, int K, uint64_t n) {
  SlotSpecies& S = s.slot;
  const size_t cap = pg.ncells() * (size_t)K;
  S.K = K;
  for (int b = 0; b < 2; ++b) {
    SPX_CUDA_TRY(cudaMalloc(&S.dx[b], cap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.dy[b], cap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.px[b], cap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.py[b], cap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.pz[b], cap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.tag[b], cap * sizeof(uint32_t)));
    SPX_CUDA_TRY(cudaMalloc(&S.nlow[b], pg.ncells() * sizeof(uint32_t)));
    SPX_CUDA_TRY(cudaMalloc(&S.ntop[b], pg.ncells() * sizeof(uint32_t)));
    SPX_CUDA_TRY(cudaMemset(S.nlow[b], 0, pg.ncells() * sizeof(uint32_t)));
    SPX_CUDA_TRY(cudaMemset(S.ntop[b], 0, pg.ncells() * sizeof(uint32_t)));
  }
  S.ocap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(1u << 16, n / 32), 1u << 28);
  for (int b = 0; b < 2; ++b) {
    SPX_CUDA_TRY(cudaMalloc(&S.ocell[b], S.ocap * sizeof(uint32_t)));
    SPX_CUDA_TRY(cudaMalloc(&S.odx[b], S.ocap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.ody[b], S.ocap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.opx[b], S.ocap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.opy[b], S.ocap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.opz[b], S.ocap * sizeof(float)));
    SPX_CUDA_TRY(cudaMalloc(&S.otag[b], S.ocap * sizeof(uint32_t)));
  }
  SPX_CUDA_TRY(cudaMalloc(&S.ocount, 2 * sizeof(uint32_t)));
  SPX_CUDA_TRY(cudaMemset(S.ocount, 0, 2 * sizeof(uint32_t)));
}

void slot_release(Species& s) {
  SlotSpecies& S = s.slot;
  for (int b = 0; b < 2; ++b) {
    for (void* p : {(void*)S.dx[b], (void*)S.dy[b], (void*)S.px[b], (void*)S.py[b], (void*)S.pz[b], (void*)S.tag[b],
                    (void*)S.nlow[b], (void*)S.ntop[b], (void*)S.ocell[b], (void*)S.odx[b], (void*)S.ody[b],
                    (void*)S.opx[b], (void*)S.opy[b], (void*)S.opz[b], (void*)S.otag[b]})
      if (p) cudaFree(p);
  }
  if (S.ocount) cudaFree(S.ocount);
  S = SlotSpecies();
}

// ---------------------------------------------------------------- plain FP32 path
// Baseline for the split path: positions are global floats x = ix + dx,
// y = iy + dy in the reference's particle order, one thread per particle,
// deposits straight into the global fields with atomics, no sorting.
__device__ __forceinline__ void plain_cell(float x, int& ix, float& dx) {
  ix = (int)floorf(x + 0.5f);
  dx = x - (float)ix;
}

__device__ __forceinline__ void plain_bc(const PhysParams& p, int nx, int ny, float& x, float& y, float& px) {
  if (y < 0.5f)
    y += (float)ny;
  else if (y >= (float)ny + 0.5f)
    y -= (float)ny;
  if (p.periodic_x) {
    if (x < 0.5f)
      x += (float)nx;
    else if (x >= (float)nx + 0.5f)
      x -= (float)nx;
  } else {
    const float wall = (float)p.wall_loc;
    if (x > wall) {  // reflect about the centre of the wall cell
      x = 2.0f * wall - x;
      px = -px;
    }
    const float lwall = (float)(p.delta + 1);
    if (p.left_wall && x < lwall) {
      x = 2.0f * lwall - x;
      px = -px;
    }
  }
}

__global__ void k_plain_move_deposit(PlainSpecies P, uint64_t n, float q, Grid g, PhysParams p, FieldPtrs f) {
  const int W = g.W;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    float x = P.x[i], y = P.y[i], px = P.px[i], py = P.py[i], pz = P.pz[i];
    const float psa = gamma_of(px, py, pz, p.csqinv);
    const float inv = 1.0f / psa;
    const float c1 = 0.5f * p.dt * inv;
    x += c1 * px;
    y += c1 * py;
    plain_bc(p, g.nx, g.ny, x, y, px);
    int ix, iy;
    float dx, dy, w[9];
    plain_cell(x, ix, dx);
    plain_cell(y, iy, dy);
    tsc_weights(dx, dy, w);
    const float vx = q * px * inv, vy = q * py * inv, vz = q * pz * inv;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) {
        const size_t o = (size_t)(iy - 1 + r) * W + (ix - 1 + k);
        atomicAdd(f.J[0] + o, w[r * 3 + k] * vx);
        atomicAdd(f.J[1] + o, w[r * 3 + k] * vy);
        atomicAdd(f.J[2] + o, w[r * 3 + k] * vz);
      }
    x += c1 * px;
    y += c1 * py;
    plain_bc(p, g.nx, g.ny, x, y, px);
    plain_cell(x, ix, dx);
    plain_cell(y, iy, dy);
    tsc_weights(dx, dy, w);
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) {
        const size_t o = (size_t)(iy - 1 + r) * W + (ix - 1 + k);
        atomicAdd(f.dsty + o, w[r * 3 + k] * q);
        atomicAdd(f.dens + o, w[r * 3 + k]);
      }
    P.x[i] = x;
    P.y[i] = y;
    P.px[i] = px;
  }
}

__global__ void k_plain_push(PlainSpecies P, uint64_t n, float beta, float alpha, Grid g, PhysParams p, FieldPtrs f) {
  const int W = g.W;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    float px = P.px[i], py = P.py[i], pz = P.pz[i];
    int ix, iy;
    float dx, dy, w[9];
    plain_cell(P.x[i], ix, dx);
    plain_cell(P.y[i], iy, dy);
    tsc_weights(dx, dy, w);
    const float* src[6] = {f.E[0], f.E[1], f.E[2], f.B[0], f.B[1], f.B[2]};
    float gth[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float* b = src[k] + (size_t)(iy - 1) * W + (ix - 1);
      float t = w[0] * __ldg(b);
      t += w[1] * __ldg(b + 1);
      t += w[2] * __ldg(b + 2);
      t += w[3] * __ldg(b + W);
      t += w[4] * __ldg(b + W + 1);
      t += w[5] * __ldg(b + W + 2);
      t += w[6] * __ldg(b + 2 * W);
      t += w[7] * __ldg(b + 2 * W + 1);
      t += w[8] * __ldg(b + 2 * W + 2);
      gth[k] = t;
    }
    float psa;
    boris(gth, beta, alpha, p.csqinv, px, py, pz, psa);
    P.px[i] = px;
    P.py[i] = py;
    P.pz[i] = pz;
  }
}

int plain_move_deposit(Species& s, uint64_t n, const ParticleGeom& pg, const PhysParams& pp, const FieldPtrs& fp,
                       int* derr, cudaStream_t st) {
  (void)derr;
  if (n) k_plain_move_deposit<<<148 * 16, 256, 0, st>>>(s.plain, n, s.charge, pg.g, pp, fp);
  SPX_CUDA_TRY(cudaGetLastError());
  return 1;
}

int plain_push(Species& s, uint64_t n, const ParticleGeom& pg, const PhysParams& pp, const FieldPtrs& fp, int* derr,
               cudaStream_t st) {
  (void)derr;
  if (n) k_plain_push<<<148 * 16, 256, 0, st>>>(s.plain, n, s.beta, s.alpha, pg.g, pp, fp);
  SPX_CUDA_TRY(cudaGetLastError());
  return 1;
}

// ---------------------------------------------------------------- diagnostics
__device__ __forceinline__ void block_add_double(double v, double* out) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, v);
}

__global__ void k_kinetic_slot(SpeciesArgs S, int TC, size_t ncells, float mass, float c, double* acc) {
  const double csq = (double)c * c;
  const float csqinv = 1.0f / (c * c);
  double e = 0, cnt = 0;
  for (size_t gc = blockIdx.x * (size_t)blockDim.x + threadIdx.x; gc < ncells; gc += (size_t)gridDim.x * blockDim.x) {
    const size_t tile = gc / TC;
    const int cc = (int)(gc - tile * TC);
    const int nlow = (int)S.nlow[gc], ntop = (int)S.ntop[gc];
    const size_t base = tile * (size_t)S.K * TC + cc;
    for (int n = 0; n < nlow + ntop; ++n) {
      const int slot = n < nlow ? n : S.K - 1 - (n - nlow);
      const size_t i = base + (size_t)slot * TC;
      const double g = (double)gamma_of(S.px[i], S.py[i], S.pz[i], csqinv);
      e += (double)mass * (g - 1.0) * csq;
      cnt += 1.0;
    }
  }
  block_add_double(e, acc);
  block_add_double(cnt, acc + 1);
}

__global__ void k_kinetic_ovf(SpeciesArgs S, float mass, float c, double* acc) {
  const uint32_t n = min(*S.rocount, S.ocap);
  const double csq = (double)c * c;
  const float csqinv = 1.0f / (c * c);
  double e = 0, cnt = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double g = (double)gamma_of(S.ropx[i], S.ropy[i], S.ropz[i], csqinv);
    e += (double)mass * (g - 1.0) * csq;
    cnt += 1.0;
  }
  block_add_double(e, acc);
  block_add_double(cnt, acc + 1);
}

__global__ void k_kinetic_plain(PlainSpecies P, uint64_t n, float mass, float c, double* acc) {
  const double csq = (double)c * c;
  const float csqinv = 1.0f / (c * c);
  double e = 0, cnt = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double g = (double)gamma_of(P.px[i], P.py[i], P.pz[i], csqinv);
    e += (double)mass * (g - 1.0) * csq;
    cnt += 1.0;
  }
  block_add_double(e, acc);
  block_add_double(cnt, acc + 1);
}

void kinetic_energy(const Species& s, const ParticleGeom& pg, bool plain, float c, double* d_acc, cudaStream_t st) {
  if (plain) {
    if (s.n) k_kinetic_plain<<<148 * 4, 256, 0, st>>>(s.plain, s.n, s.mass, c, d_acc);
  } else {
    SpeciesArgs A = species_args(const_cast<Species&>(s));
    k_kinetic_slot<<<148 * 4, 256, 0, st>>>(A, pg.TC(), pg.ncells(), s.mass, c, d_acc);
    k_kinetic_ovf<<<16, 256, 0, st>>>(A, s.mass, c, d_acc);
  }
  SPX_CUDA_TRY(cudaGetLastError());
}

// ---------------------------------------------------------------- seeded initialisation
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011), written from the published
// round function and constants.
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    const uint32_t hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return ctr;
}
__device__ __forceinline__ float u01_open0(uint32_t x) { return ((x >> 8) + 1u) * (1.0f / 16777216.0f); }  // (0,1]
__device__ __forceinline__ float u01(uint32_t x) { return (x >> 8) * (1.0f / 16777216.0f); }               // [0,1)

__global__ void k_init(InitSpec is, int ny, uint64_t n, uint32_t* cell, float* dxo, float* dyo, float* pxo,
                       float* pyo, float* pzo) {
  const int ncols = is.x1 - is.x0;
  const float c = is.c;
  const float csqinv = 1.0f / (c * c);
  const float g = is.gamma_drift;
  const float beta_inj = g > 1.0f ? is.sign_x * sqrtf(1.0f - 1.0f / (g * g)) : 0.0f;  // src/prtls.rs:224
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)(i % is.ppc);
    const uint64_t cidx = i / is.ppc;
    const int col = is.x0 + (int)(cidx % ncols), row = (int)(cidx / ncols);
    const uint2 key = make_uint2((uint32_t)is.seed, (uint32_t)(is.seed >> 32));
    const uint4 r0 = philox4x32_10(make_uint4((uint32_t)i, (uint32_t)(i >> 32), 0u, 0x5eed0001u), key);
    const uint4 r1 = philox4x32_10(make_uint4((uint32_t)i, (uint32_t)(i >> 32), 1u, 0x5eed0001u), key);
    float dx, dy;
    if (is.random_positions) {
      dx = u01(r1.z) - 0.5f;
      dy = u01(r1.w) - 0.5f;
    } else {  // src/prtls.rs:209-212
      float r = 1.0f / (2.0f * (float)is.ppc);
      r += (float)k / (float)is.ppc;
      dx = r - 0.5f;
      dy = r - 0.5f;
    }
    // Box-Muller normals
    const float ra = sqrtf(-2.0f * logf(u01_open0(r0.x))), rb = sqrtf(-2.0f * logf(u01_open0(r0.z)));
    float sa, ca, sb, cb;
    sincospif(2.0f * u01(r0.y), &sa, &ca);
    sincospif(2.0f * u01(r0.w), &sb, &cb);
    const float n1 = ra * ca, n2 = ra * sa, n3 = rb * cb;
    const float uflip = u01(r1.x);
    // src/prtls.rs:231-249
    float px = n1 * (is.vth * c), py = n2 * (is.vth * c), pz = n3 * (is.vth * c);
    float psa = sqrtf(1.0f + (px * px + py * py + pz * pz) * csqinv);
    if (g > 1.0f) {
      float ux = px / c;
      if (-beta_inj * ux > uflip * psa) ux *= -1.0f;
      px = g * (ux + beta_inj * psa);
      px *= c;
    }
    const int ix = col + 1, iy = row + 1;
    cell[i] = (uint32_t)ix | ((uint32_t)iy << 16);
    dxo[i] = dx;
    dyo[i] = dy;
    pxo[i] = px;
    pyo[i] = py;
    pzo[i] = pz;
  }
}

void init_particles(const InitSpec& is, const Grid& g, uint64_t n, uint32_t* cell, float* dx, float* dy, float* px,
                    float* py, float* pz, cudaStream_t st) {
  if (n) k_init<<<148 * 16, 256, 0, st>>>(is, g.ny, n, cell, dx, dy, px, py, pz);
  SPX_CUDA_TRY(cudaGetLastError());
}

}  // namespace spx
