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

// ---------------------------------------------------------------- packed FP32x2
// sm_100a executes two FP32 operations per instruction (add/sub/mul/fma .f32x2).
// A lone packed mul, add or sub rounds each element exactly like the scalar
// .rn operation, but the code generator fuses a packed multiply feeding a
// packed add into a fused multiply-add even with contraction disabled (measured:
// ~26% of random mul+add pairs differ from the scalar result).  So on the exact
// path a packed product never feeds a packed sum: packed products are summed
// with scalar adds, or scalar products with packed adds (both measured
// bit-identical to the scalar chain over 2^20 random inputs).  Fused packed
// multiply-adds appear only in the deposit sums, whose order and rounding are
// not the reference's anyway.
__device__ __forceinline__ unsigned long long pk2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 up2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return up2(r);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return up2(r);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)));
  return up2(r);
}
// fused multiply-add: only for sums whose rounding is not the reference's anyway (deposits)
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
  return up2(r);
}
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

// tsc_weights restated pairwise: w00/w02, w20/w22 and w10/w12 share their
// left factors and differ only in (0.5 - dx) vs (0.5 + dx), so each pair is
// one packed product chain with the reference's association order.  The two
// 0.75 - d*d terms (a multiply feeding a subtraction) stay scalar.
__device__ __forceinline__ void tsc_weights_x2(float dx, float dy, float (&w)[9]) {
  const float2 ab = sub2(bc2(0.5f), make_float2(dy, -dy));  // (0.5 - dy, 0.5 + dy)
  const float2 cd = sub2(bc2(0.5f), make_float2(dx, -dx));  // (0.5 - dx, 0.5 + dx)
  const float2 p1 = mul2(bc2(0.5f), ab);
  const float2 p2 = mul2(p1, ab);                             // (0.5 a a, 0.5 b b)
  const float2 p3 = mul2(p2, bc2(0.5f));
  const float2 fh = make_float2(0.75f - dy * dy, 0.75f - dx * dx);
  const float f05 = fh.x * 0.5f;
  const float2 r0 = mul2(mul2(bc2(p3.x), cd), cd);  // w00, w02
  const float2 r1 = mul2(mul2(bc2(f05), cd), cd);   // w10, w12
  const float2 r2 = mul2(mul2(bc2(p3.y), cd), cd);  // w20, w22
  const float2 m = mul2(p2, bc2(fh.y));             // w01, w21
  w[0] = r0.x;
  w[1] = m.x;
  w[2] = r0.y;
  w[3] = r1.x;
  w[4] = fh.x * fh.y;
  w[5] = r1.y;
  w[6] = r2.x;
  w[7] = m.y;
  w[8] = r2.y;
}

// TSC weights are quadratics of the offset d (src/lib.rs:339-347):
//   W0 = 0.5 (0.5 - d)^2 = 1/8 - d/2 + d^2/2,  W1 = 3/4 - d^2,  W2 = 1/8 + d/2 + d^2/2,
// so the stencil a cell's particles deposit, S[a][b] = sum_p v_p W_a(dy_p) W_b(dx_p),
// is fixed by the nine moments M[i][j] = sum_p v_p dy_p^i dx_p^j (i, j = 0..2):
// S[a][b] = sum_ij P[a][i] P[b][j] M[i][j].  A particle then adds to nine
// moments instead of evaluating nine weights, and the stencil is formed once per
// cell.  (Deposit sums are not in the reference's order anyway, so only their
// rounding changes: a few ulps of the cell's total.)
__device__ __forceinline__ float tsc_poly(int a, int i) {
  // rows: W0, W1, W2; columns: coefficient of d^0, d^1, d^2
  return a == 1 ? (i == 0 ? 0.75f : i == 1 ? 0.f : -1.f) : (i == 0 ? 0.125f : i == 2 ? 0.5f : (a == 0 ? -0.5f : 0.5f));
}
// m[i*3 + j] (dy power i, dx power j) -> s[a*3 + b] (stencil row a = y offset, column b = x offset)
__device__ __forceinline__ void moments_to_stencil(const float (&m)[9], float (&s)[9]) {
  // the zero coefficient of W1 is skipped (indices are compile-time after unrolling)
  auto dot3 = [](int row, float x0, float x1, float x2) {
    float r = tsc_poly(row, 0) * x0 + tsc_poly(row, 2) * x2;
    return row == 1 ? r : r + tsc_poly(row, 1) * x1;
  };
  float n[9];  // n[i*3 + b] = sum_j P[b][j] m[i*3 + j]
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int b = 0; b < 3; ++b) n[i * 3 + b] = dot3(b, m[i * 3], m[i * 3 + 1], m[i * 3 + 2]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) s[a * 3 + b] = dot3(a, n[b], n[3 + b], n[6 + b]);
}

// Boris push of src/prtls.rs:412-440 given the gathered fields g[0..5] = E, B.
// Every operation is the reference's, in its order (Rust evaluates a + b * c - d * e
// as (a + (b*c)) - (d*e)).  Scalar: its products pair operands in ever different
// combinations, and packing them cost more register moves than it saved (measured:
// 0.7 % more instructions per particle with packed products).
__device__ __forceinline__ void boris(const float (&g)[6], float beta, float alpha, float csqinv, float& px,
                                      float& py, float& pz, float& psa) {
  const float ext = g[0] * beta, eyt = g[1] * beta, ezt = g[2] * beta;
  const float bx0 = g[3] * alpha, by0 = g[4] * alpha;
  const float ux = px + ext, uy = py + eyt, uz = pz + ezt;
  const float gt = 1.0f / sqrtf(1.0f + (ux * ux + uy * uy + uz * uz) * csqinv);
  const float bxt = bx0 * gt, byt = by0 * gt, bzt = (g[5] * alpha) * gt;
  const float boris = 2.0f * (1.0f / (1.0f + bxt * bxt + byt * byt + bzt * bzt));
  // u' = u + u x B
  const float uxt = ux + uy * bzt - uz * byt;
  const float uyt = uy + uz * bxt - ux * bzt;
  const float uzt = uz + ux * byt - uy * bxt;
  // p = u + boris (u' x B) + E
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
  const float2 d = make_float2(c1 * px, c1 * py);
  dx += d.x;
  if (dx >= 0.5f) {
    dx -= 1.0f;
    ix += 1;
  } else if (dx < -0.5f) {
    dx += 1.0f;
    ix -= 1;
  }
  dy += d.y;
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
// the x part of apply_bc without the periodic feature: the reflecting wall
__device__ __forceinline__ void wall_x(const PhysParams& p, int& ix, float& dx, float& px, int* derr) {
  {
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
    wall_x(p, ix, dx, px, derr);
  }
}

// ---------------------------------------------------------------- split path kernel
struct SpeciesArgs {
  float *dx, *dy, *px, *py, *pz;
  uint32_t* tag;
  uint32_t* nlow;  // low range extents: rewritten by each cell's owner during a moving step
  uint32_t* ain;   // entries of the arrival region read this step (emptied by the owner)
  uint32_t* aout;  // entries of the arrival region written this step (atomic)
  // overflow lists: read (r*) and write (w*)
  const uint32_t* rocell;
  float *rodx, *rody, *ropx, *ropy, *ropz;
  const uint32_t* rotag;
  uint32_t* wocell;
  float *wodx, *wody, *wopx, *wopy, *wopz;
  uint32_t* wotag;
  const uint32_t* rocount;
  uint32_t* wocount;
  uint32_t ocap;
  float charge, alpha, beta;
  int K, KL, H;
  int rin, rout;  // first slot of the region read / written
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

// Park a particle in the overflow list (no room in its cell); the fallback
// kernel advances it with the rest until the host repacks.
__device__ __forceinline__ void park(const StepArgs& a, const SpeciesArgs& S, int ix, int iy, float dx, float dy,
                                     float px, float py, float pz, uint32_t tag) {
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

// Append a particle that left its cell (or found its low range full) to the
// arrival region written this step: entry i of the destination's region, i
// from its arrivals counter.  The owner of the destination reads another
// region and writes only below KL, so the append never meets its accesses.
__device__ __forceinline__ void relocate(const StepArgs& a, const SpeciesArgs& S, int ix, int iy, float dx, float dy,
                                         float px, float py, float pz, uint32_t tag) {
  const int TC = a.TX * a.TY;
  const int dtx = (ix - 1) >> a.logTX, dty = (iy - 1) >> a.logTY;
  const int dc = (((iy - 1) & (a.TY - 1)) << a.logTX) | ((ix - 1) & (a.TX - 1));
  const size_t dtile = (size_t)dty * a.NTX + dtx;
  const size_t dgc = dtile * TC + dc;
  const int i = (int)atomicAdd(&S.aout[dgc], 1u);
  if (i < S.H) {
    const size_t widx = dtile * (size_t)S.K * TC + (size_t)(S.rout + i) * TC + dc;
    S.dx[widx] = dx;
    S.dy[widx] = dy;
    S.px[widx] = px;
    S.py[widx] = py;
    S.pz[widx] = pz;
    S.tag[widx] = tag;
  } else {
    atomicSub(&S.aout[dgc], 1u);
    park(a, S, ix, iy, dx, dy, px, py, pz, tag);
  }
}

// E/B window of a tile in shared memory: (TY+2) x (TX+2) cells, one float4
// {Ex, Ey, Ez, Bx} and one float2 {By, Bz} per cell, so a gather of one
// neighbour cell is two vector loads.  A 128-bit load is served 8 lanes per
// wavefront and a 64-bit load 16 lanes per wavefront; the lanes of a warp own
// consecutive cells of a tile row, so both are conflict-free.
__host__ __device__ inline size_t eb_floats(int TX, int TY) { return (size_t)6 * (TX + 2) * (TY + 2); }

// Per-warp queues of the rare work (a particle whose half-step cell differs
// from its owner cell deposits J elsewhere; a particle whose full-step cell
// differs deposits rho elsewhere and moves to another cell).  Lanes append with
// a ballot; the warp drains a queue cooperatively once it holds >= 32 entries,
// so the rare paths run converged instead of as divergent branches.
constexpr int QCAP = 64;     // entries per queue
constexpr int QWORDS = 7;    // words per entry
constexpr int QWARP = 2 * QWORDS * QCAP;  // floats per warp (J queue + mover queue)
// Deposit window planes: Jx, Jy, Jz, rho, dens, then (compensated sums) the
// compensation terms of Jx, Jy, Jz.
__host__ __device__ inline int win_planes(bool move, bool comp) { return move ? (comp ? 8 : 5) : 0; }
__host__ __device__ inline size_t slot_smem_floats(int TX, int TY, bool push, bool move, bool comp = false) {
  const size_t win = (size_t)win_planes(move, comp) * (TX + 4) * (TY + 4);
  const size_t eb = push ? eb_floats(TX, TY) : 0;
  const size_t q = move ? (size_t)(TX * TY / 32) * QWARP : 0;
  return win + eb + q;
}

// The queue drains run rarely (once per ~32 queued particles of a warp); as
// separate functions they keep their registers out of the main loop's budget.
__device__ __noinline__ void drain_j_fn(const StepArgs& a, const float* qj, int nq, int lane, float* win, int WX,
                                        int WY, int wx0, int wy0) {
  const int WN = WX * WY, W = a.g.W;
  for (int e = lane; e < nq; e += 32) {
    const uint32_t cell = __float_as_uint(qj[0 * QCAP + e]);
    const int jx = (int)(cell & 0xFFFFu), jy = (int)(cell >> 16);
    float w[9];
    tsc_weights(qj[1 * QCAP + e], qj[2 * QCAP + e], w);
    dep9(win, WX, WY, wx0, wy0, a.f.J[0], W, jx, jy, w, qj[3 * QCAP + e]);
    dep9(win + WN, WX, WY, wx0, wy0, a.f.J[1], W, jx, jy, w, qj[4 * QCAP + e]);
    dep9(win + 2 * WN, WX, WY, wx0, wy0, a.f.J[2], W, jx, jy, w, qj[5 * QCAP + e]);
  }
  __syncwarp();
}
__device__ __noinline__ void drain_m_fn(const StepArgs& a, const SpeciesArgs& S, const float* qm, int nq, int lane,
                                        float* win, int WX, int WY, int wx0, int wy0, float q) {
  const int WN = WX * WY, W = a.g.W;
  for (int e = lane; e < nq; e += 32) {
    const uint32_t cell = __float_as_uint(qm[0 * QCAP + e]);
    const int mx = (int)(cell & 0xFFFFu), my = (int)(cell >> 16);
    const float mdx = qm[1 * QCAP + e], mdy = qm[2 * QCAP + e];
    float w[9];
    tsc_weights(mdx, mdy, w);
    dep9(win + 3 * WN, WX, WY, wx0, wy0, a.f.dsty, W, mx, my, w, q);
    dep9(win + 4 * WN, WX, WY, wx0, wy0, a.f.dens, W, mx, my, w, 1.0f);
    relocate(a, S, mx, my, mdx, mdy, qm[3 * QCAP + e], qm[4 * QCAP + e], qm[5 * QCAP + e],
             __float_as_uint(qm[6 * QCAP + e]));
  }
  __syncwarp();
}

// One CTA per tile, one thread per cell.  Every particle a thread processes
// starts in the thread's cell: E/B of the tile (+1 halo) is staged once in
// shared memory and gathered with conflict-free loads; J and rho deposits that
// stay in the owner cell's stencil accumulate in registers.  The warp walks its
// cells' slots in lock-step rounds (low range, then the arrival region), so
// the loads of a round are coalesced; the particles that stay are written back
// densely from slot 0 (a round's stores cover a few neighbouring slot rows and
// merge in L2).
#ifndef SPX_SLOT_MIN_BLOCKS
#define SPX_SLOT_MIN_BLOCKS 2  // resident 256-thread CTAs per SM the register budget is sized for
#endif
// 8x8 tiles (64-thread CTAs): ten resident CTAs per SM, i.e. 96 registers and 20 warps
// per SM instead of 128 registers and 16 warps (measured: the batch kernel 7 % faster on
// the ensemble; the few spilled values are outside the round loop's hot path)
#ifndef SPX_SLOT8_MIN_BLOCKS
#define SPX_SLOT8_MIN_BLOCKS 10
#endif
// 16x8 tiles (128-thread CTAs, tile code 168): five per SM, the same 96 registers and 20 warps
#define SPX_SLOT_BOUNDS(TS)                                      \
  __launch_bounds__((TS) == 8 ? 64 : (TS) == 168 ? 128 : 256,    \
                    (TS) == 8 ? SPX_SLOT8_MIN_BLOCKS : (TS) == 168 ? SPX_SLOT8_MIN_BLOCKS / 2 : SPX_SLOT_MIN_BLOCKS)
// apply_bc of a grid periodic in x as well as y (the reference's `periodic`
// feature) when the kernel knows it at compile time.
__device__ __forceinline__ void periodic_bc(int nx, int ny, int& ix, int& iy) {
  if (iy < 1)
    iy += ny;
  else if (iy > ny)
    iy -= ny;
  if (ix < 1)
    ix += nx;
  else if (ix > nx)
    ix -= nx;
}

// Boundary handling known at compile time: BC_ANY reads a.p, BC_PERIODIC is the
// reference's `periodic` feature, BC_WALL the reflecting wall.
enum : int { BC_ANY = 0, BC_PERIODIC = 1, BC_WALL = 2 };
template <int BC>
__device__ __forceinline__ void bc_of(const StepArgs& a, int nx, int ny, int& ix, int& iy, float& dx, float& px) {
  if (BC == BC_PERIODIC) {
    periodic_bc(nx, ny, ix, iy);
  } else if (BC == BC_WALL) {
    if (iy < 1)
      iy += ny;
    else if (iy > ny)
      iy -= ny;
    wall_x(a.p, ix, dx, px, a.derr);
  } else {
    if (iy < 1)
      iy += ny;
    else if (iy > ny)
      iy -= ny;
    if (a.p.periodic_x) {
      if (ix < 1)
        ix += nx;
      else if (ix > nx)
        ix -= nx;
    } else {
      wall_x(a.p, ix, dx, px, a.derr);
    }
  }
}

// BC: see bc_of.  TS: the tile shape known at compile time (16: 16x16, 8: 8x8, 168: 16x8; the
// index arithmetic folds), 0: the tile shape from a.
// Species [s0, s1) of the step (all of them, or one per CTA when a small grid
// splits the species across CTAs).
template <bool PUSH, bool MOVE, bool COMP = false, int BC = BC_ANY, int TS = 0>
__device__ __forceinline__ void slot_tile(const StepArgs& a, const int tile, float* smem, const int s0,
                                          const int s1) {
  constexpr int TSX = TS == 168 ? 16 : TS, TSY = TS == 168 ? 8 : TS;
  const int TXc = TSX ? TSX : a.TX, TYc = TSY ? TSY : a.TY, logTXc = TSX == 16 ? 4 : TSX == 8 ? 3 : a.logTX;
  const int TC = TXc * TYc;
  const int tx = tile % a.NTX, ty = tile / a.NTX;
  const int c = threadIdx.x;
  const int lane = c & 31, warp = c >> 5;
  const int lx = c & (TXc - 1), ly = c >> logTXc;
  const int ox = tx * TXc + lx + 1, oy = ty * TYc + ly + 1;  // owner cell (reference coords)
  const int W = a.g.W, nx = a.g.nx, ny = a.g.ny;
  // A particle moves at most one cell per half step (update_position, src/prtls.rs:103-119),
  // so the tile's particles end this step within two cells of it: when that band stays
  // inside the grid and clear of the walls, apply_bc (src/prtls.rs:124-190) is the
  // identity for all of them (and its assertion cannot fire).
  bool inner_tile;
  {
    const int X0 = tx * TXc + 1, X1 = X0 + TXc - 1, Y0 = ty * TYc + 1, Y1 = Y0 + TYc - 1;
    const bool px_ = BC == BC_PERIODIC || (BC == BC_ANY && a.p.periodic_x);
    const bool in_x = px_ ? (X0 - 2 >= 1 && X1 + 2 <= nx) : (X0 - 2 >= a.p.delta + 2 && X1 + 2 <= a.p.wall_loc - 1);
    inner_tile = in_x && Y0 - 2 >= 1 && Y1 + 2 <= ny;
  }
  // deposit window: tile + 2 cells
  const int WX = TXc + 4, WY = TYc + 4, WN = WX * WY;
  const int wx0 = tx * TXc + 1 - 2, wy0 = ty * TYc + 1 - 2;
  float* win = smem;
  float* wjx = win;
  float* wjy = win + WN;
  float* wjz = win + 2 * WN;
  float* wrho = win + 3 * WN;
  float* wdens = win + 4 * WN;
  constexpr int NWP = MOVE ? (COMP ? 8 : 5) : 0;  // deposit window planes
  // E/B window: tile + 1 cell
  const int EX = TXc + 2, EY = TYc + 2;
  float4* eb4 = reinterpret_cast<float4*>(smem + NWP * WN);  // 16-byte aligned: WN is a multiple of 4
  float2* eb2 = reinterpret_cast<float2*>(eb4 + EX * EY);
  float* after_eb = smem + NWP * WN + (PUSH ? 6 * EX * EY : 0);
  float* qbase = after_eb + warp * QWARP;
  float* qj = qbase;                   // [QWORDS][QCAP]
  float* qm = qbase + QWORDS * QCAP;   // [QWORDS][QCAP]
  if (MOVE)
    for (int i = c; i < NWP * WN; i += TC) win[i] = 0.f;
  if (PUSH) {
    // thread c stages window cells c, c + TC, ...: its (row, column) advances without divisions
    const int s_r = TC / EX, s_q = TC - s_r * EX;
    int r = c / EX, q = c - (c / EX) * EX;
    for (int i = c; i < EY * EX; i += TC) {
      const size_t g = (size_t)(ty * TYc + r) * W + (tx * TXc + q);
      eb4[i] = make_float4(__ldg(a.f.E[0] + g), __ldg(a.f.E[1] + g), __ldg(a.f.E[2] + g), __ldg(a.f.B[0] + g));
      eb2[i] = make_float2(__ldg(a.f.B[1] + g), __ldg(a.f.B[2] + g));
      q += s_q;
      r += s_r;
      if (q >= EX) {
        q -= EX;
        ++r;
      }
    }
  }
  __syncthreads();
  const int ebo = ly * EX + lx;  // top-left of this cell's 3x3 neighbourhood
  float2 accJxy[9];
  float accJz[9];
  float2 cmpJxy[9];  // compensation terms (COMP): the low-order bits the running sums lost
  float cmpJz[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    accJxy[k] = make_float2(0.f, 0.f);
    accJz[k] = 0.f;
    cmpJxy[k] = make_float2(0.f, 0.f);
    cmpJz[k] = 0.f;
  }
  const size_t gc = (size_t)tile * TC + c;
  const float half_dt = 0.5f * a.p.dt;
  const float csqinv = a.p.csqinv;
  const unsigned lt_mask = (1u << lane) - 1u;

  for (int s = s0; s < s1; ++s) {
    const SpeciesArgs& S = a.sp[s];
    const int K = S.K;
    const size_t tb = (size_t)tile * K * TC;  // this tile's block of slots
    float* __restrict__ sdx = S.dx + tb;
    float* __restrict__ sdy = S.dy + tb;
    float* __restrict__ spx = S.px + tb;
    float* __restrict__ spy = S.py + tb;
    float* __restrict__ spz = S.pz + tb;
    uint32_t* __restrict__ stg = S.tag + tb;
    const int nlow = (int)S.nlow[gc], nin = (int)S.ain[gc];
    // each lane walks its low range and then its arrivals without a gap: the warp runs
    // max(nlow + nin) rounds instead of max(nlow) + max(nin)
    const int rounds = __reduce_max_sync(0xffffffffu, nlow + nin);
    const int KL = S.KL, rin = S.rin;
    int kept = 0;  // particles kept so far (moving steps): the next low-range slot
    const float q = S.charge, beta = S.beta, alpha = S.alpha;
    // density moments of the particles that stay (the count is `kept`):
    // rm1 = (sum dx, sum dy), rm2 = (sum dx^2, sum dy^2), rm11 = sum dx dy,
    // rm12 = (sum dy dx^2, sum dx dy^2), rm22 = sum dx^2 dy^2
    float2 rm1 = make_float2(0.f, 0.f), rm2 = make_float2(0.f, 0.f), rm12 = make_float2(0.f, 0.f);
    float rm11 = 0.f, rm22 = 0.f;
    int nq_j = 0, nq_m = 0;  // warp-uniform queue sizes

    auto slot_of = [&](int r, bool& act) -> int {
      act = r < nlow + nin;
      return r < nlow ? r : rin + (r - nlow);
    };
    // drain the J queue: deposit the stencils whose centre left the owner cell
    auto drain_j = [&]() {
      drain_j_fn(a, qj, nq_j, lane, win, WX, WY, wx0, wy0);
      nq_j = 0;
    };
    // drain the mover queue: rho/dens at the new cell, then relocation
    auto drain_m = [&]() {
      drain_m_fn(a, S, qm, nq_m, lane, win, WX, WY, wx0, wy0, q);
      nq_m = 0;
    };

    // software pipeline: the state of round r+1 is loaded during round r (with
    // the tag on moving steps: a particle that moves or shifts down takes it along)
    float ndx = 0.f, ndy = 0.f, npx = 0.f, npy = 0.f, npz = 0.f;
    uint32_t ntg = 0u;
    bool nact = false;
    int nidx = c;
    if (rounds > 0) {
      const int sl = slot_of(0, nact);
      nidx = sl * TC + c;
      if (nact) {
        ndx = sdx[nidx];
        ndy = sdy[nidx];
        npx = spx[nidx];
        npy = spy[nidx];
        npz = spz[nidx];
        if (MOVE) ntg = stg[nidx];
      }
    }
    for (int r = 0; r < rounds; ++r) {
      const int idx = nidx;
      const bool act = nact;
      float dx = ndx, dy = ndy, px = npx, py = npy, pz = npz;
      const uint32_t tg = ntg;
      if (r + 1 < rounds) {
        const int sl = slot_of(r + 1, nact);
        nidx = sl * TC + c;
        if (nact) {
          ndx = sdx[nidx];
          ndy = sdy[nidx];
          npx = spx[nidx];
          npy = spy[nidx];
          npz = spz[nidx];
          if (MOVE) ntg = stg[nidx];
        }
      }
      bool jcross = false, mover = false;
      int ix = ox, iy = oy, jxc = ox, jyc = oy;
      float jdx = 0.f, jdy = 0.f, vx = 0.f, vy = 0.f, vz = 0.f;
      if (act) {
        float psa;
        if (PUSH) {
          float w[9];
          tsc_weights_x2(dx, dy, w);
          // six running sums, neighbour cells in the reference's order w00 .. w22
          float gth[6];
          float2 g01, g23, g45;
#pragma unroll
          for (int k = 0; k < 9; ++k) {
            const int o = ebo + (k / 3) * EX + (k % 3);
            const float4 e4 = eb4[o];
            const float2 e2 = eb2[o];
            const float2 p01 = make_float2(w[k] * e4.x, w[k] * e4.y);
            const float2 p23 = make_float2(w[k] * e4.z, w[k] * e4.w);
            const float2 p45 = make_float2(w[k] * e2.x, w[k] * e2.y);
            if (k == 0) {
              g01 = p01; g23 = p23; g45 = p45;
            } else {
              g01 = add2(g01, p01); g23 = add2(g23, p23); g45 = add2(g45, p45);
            }
          }
          gth[0] = g01.x; gth[1] = g01.y; gth[2] = g23.x; gth[3] = g23.y; gth[4] = g45.x; gth[5] = g45.y;
          boris(gth, beta, alpha, csqinv, px, py, pz, psa);
        } else {
          psa = gamma_of(px, py, pz, csqinv);
        }
        if (!MOVE) {
          spx[idx] = px;
          spy[idx] = py;
          spz[idx] = pz;
        } else {
          const float inv = 1.0f / psa;
          const float c1 = half_dt * inv;
          // first half: position, boundaries, current (src/lib.rs:480-484)
          move_half(c1, px, py, ix, iy, dx, dy);
          if (!inner_tile) bc_of<BC>(a, nx, ny, ix, iy, dx, px);
          {
            vx = (q * px) * inv;
            vy = (q * py) * inv;
          }
          vz = q * pz * inv;
          jcross = ix != ox || iy != oy;
          if (!jcross && !COMP) {
            // moments sum v dy^i dx^j, i, j = 0..2 (see moments_to_stencil); fused
            // multiply-adds: the deposit sums are not the reference's order anyway
            const float2 vxy = make_float2(vx, vy);
            const float2 a1 = mul2(vxy, bc2(dx));  // v dx
            const float2 a2 = mul2(a1, bc2(dx));   // v dx^2
            const float z1 = vz * dx, z2 = z1 * dx;
            const float dy2 = dy * dy;
            accJxy[0] = add2(accJxy[0], vxy);
            accJxy[1] = add2(accJxy[1], a1);
            accJxy[2] = add2(accJxy[2], a2);
            accJxy[3] = fma2(bc2(dy), vxy, accJxy[3]);
            accJxy[4] = fma2(bc2(dy), a1, accJxy[4]);
            accJxy[5] = fma2(bc2(dy), a2, accJxy[5]);
            accJxy[6] = fma2(bc2(dy2), vxy, accJxy[6]);
            accJxy[7] = fma2(bc2(dy2), a1, accJxy[7]);
            accJxy[8] = fma2(bc2(dy2), a2, accJxy[8]);
            accJz[0] += vz;
            accJz[1] += z1;
            accJz[2] += z2;
            accJz[3] = __fmaf_rn(dy, vz, accJz[3]);
            accJz[4] = __fmaf_rn(dy, z1, accJz[4]);
            accJz[5] = __fmaf_rn(dy, z2, accJz[5]);
            accJz[6] = __fmaf_rn(dy2, vz, accJz[6]);
            accJz[7] = __fmaf_rn(dy2, z1, accJz[7]);
            accJz[8] = __fmaf_rn(dy2, z2, accJz[8]);
          } else if (!jcross) {
            float w[9];
            tsc_weights_x2(dx, dy, w);
            const float2 vxy = make_float2(vx, vy);
#pragma unroll
            for (int k = 0; k < 9; ++k) {
              {  // Kahan summation: y = w v - comp; t = acc + y; comp = (t - acc) - y
                const float2 y = fma2(bc2(w[k]), vxy, make_float2(-cmpJxy[k].x, -cmpJxy[k].y));
                const float2 t = add2(accJxy[k], y);
                cmpJxy[k] = sub2(sub2(t, accJxy[k]), y);
                accJxy[k] = t;
                const float yz = __fmaf_rn(w[k], vz, -cmpJz[k]);
                const float tz = __fadd_rn(accJz[k], yz);
                cmpJz[k] = __fsub_rn(__fsub_rn(tz, accJz[k]), yz);
                accJz[k] = tz;
              }
            }
          } else {
            jxc = ix;
            jyc = iy;
            jdx = dx;
            jdy = dy;
          }
          // second half: position, boundaries, density (src/lib.rs:486-488)
          move_half(c1, px, py, ix, iy, dx, dy);
          if (!inner_tile) bc_of<BC>(a, nx, ny, ix, iy, dx, px);
          // a particle that stays but finds the low range full joins its own
          // cell's arrivals like a mover
          mover = ix != ox || iy != oy || kept >= KL;
          if (!mover) {
            // density moments (the count is `kept`): sum dx, dy, dx^2, dy^2, dx dy, dy dx^2, dx dy^2, dx^2 dy^2
            const float2 dd = make_float2(dx, dy);
            const float2 sq = mul2(dd, dd);
            rm1 = add2(rm1, dd);
            rm2 = add2(rm2, sq);
            rm11 = __fmaf_rn(dx, dy, rm11);
            rm12 = fma2(make_float2(dy, dx), sq, rm12);
            rm22 = __fmaf_rn(sq.x, sq.y, rm22);
            const int o = kept * TC + c;
            sdx[o] = dx;
            sdy[o] = dy;
            spx[o] = px;
            spy[o] = py;
            spz[o] = pz;
            if (o != idx) stg[o] = tg;
            ++kept;
          }
        }
      }
      if (MOVE) {
        const unsigned mj = __ballot_sync(0xffffffffu, jcross);
        if (mj) {
          if (jcross) {
            const int e = nq_j + __popc(mj & lt_mask);
            qj[0 * QCAP + e] = __uint_as_float((uint32_t)jxc | ((uint32_t)jyc << 16));
            qj[1 * QCAP + e] = jdx;
            qj[2 * QCAP + e] = jdy;
            qj[3 * QCAP + e] = vx;
            qj[4 * QCAP + e] = vy;
            qj[5 * QCAP + e] = vz;
          }
          nq_j += __popc(mj);
          __syncwarp();
          if (nq_j >= 32) drain_j();
        }
        const unsigned mm = __ballot_sync(0xffffffffu, mover);
        if (mm) {
          if (mover) {
            const int e = nq_m + __popc(mm & lt_mask);
            qm[0 * QCAP + e] = __uint_as_float((uint32_t)ix | ((uint32_t)iy << 16));
            qm[1 * QCAP + e] = dx;
            qm[2 * QCAP + e] = dy;
            qm[3 * QCAP + e] = px;
            qm[4 * QCAP + e] = py;
            qm[5 * QCAP + e] = pz;
            qm[6 * QCAP + e] = __uint_as_float(tg);
          }
          nq_m += __popc(mm);
          __syncwarp();
          if (nq_m >= 32) drain_m();
        }
      }
    }
    if (MOVE) {
      if (nq_j) drain_j();
      if (nq_m) drain_m();
      S.nlow[gc] = (uint32_t)kept;
      S.ain[gc] = 0u;
      // this species' density stencil of the owner cell -> window
      if (kept > 0) {
        const float m[9] = {(float)kept, rm1.x, rm2.x, rm1.y, rm11, rm12.x, rm2.y, rm12.y, rm22};
        float d[9];
        moments_to_stencil(m, d);
        const int bl = (oy - 1 - wy0) * WX + (ox - 1 - wx0);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            atomicAdd(wrho + bl + r * WX + k, d[r * 3 + k] * q);
            atomicAdd(wdens + bl + r * WX + k, d[r * 3 + k]);
          }
      }
    }
  }
  if (!MOVE) return;
  if (!COMP) {  // the current moments -> stencils (accumulated in place)
    float mx[9], my[9], mz[9], sx[9], sy[9], sz[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      mx[k] = accJxy[k].x;
      my[k] = accJxy[k].y;
      mz[k] = accJz[k];
    }
    moments_to_stencil(mx, sx);
    moments_to_stencil(my, sy);
    moments_to_stencil(mz, sz);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      accJxy[k] = make_float2(sx[k], sy[k]);
      accJz[k] = sz[k];
    }
  }
  {
    const int bl = (oy - 1 - wy0) * WX + (ox - 1 - wx0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        atomicAdd(wjx + bl + r * WX + k, accJxy[r * 3 + k].x);
        atomicAdd(wjy + bl + r * WX + k, accJxy[r * 3 + k].y);
        atomicAdd(wjz + bl + r * WX + k, accJz[r * 3 + k]);
        if (COMP) {  // the compensation travels with the tile flush
          atomicAdd(win + 5 * WN + bl + r * WX + k, -cmpJxy[r * 3 + k].x);
          atomicAdd(win + 6 * WN + bl + r * WX + k, -cmpJxy[r * 3 + k].y);
          atomicAdd(win + 7 * WN + bl + r * WX + k, -cmpJz[r * 3 + k]);
        }
      }
  }
  __syncthreads();
  // window -> global (clipped to the ghosted grid): thread c flushes cells c, c + TC, ... of
  // each plane, its (row, column) advanced without divisions
  const int s_wy = TC / WX, s_wx = TC - s_wy * WX;
  const int c_wy = c / WX, c_wx = c - c_wy * WX;
#pragma unroll 1
  for (int plane = 0; plane < 5; ++plane) {
    float* d = plane == 0 ? a.f.J[0] : plane == 1 ? a.f.J[1] : plane == 2 ? a.f.J[2] : plane == 3 ? a.f.dsty : a.f.dens;
    const float* wp = win + plane * WN;
    int wx = c_wx, wy = c_wy;
    for (int k = c; k < WN; k += TC) {
      float v = wp[k];
      if (COMP && plane < 3) v += wp[k + 5 * WN];  // one rounding of sum + compensation
      const int gx = wx0 + wx, gy = wy0 + wy;
      if (v != 0.f && gx >= 0 && gx <= nx + 1 && gy >= 0 && gy <= ny + 1) atomicAdd(d + (size_t)gy * W + gx, v);
      wx += s_wx;
      wy += s_wy;
      if (wx >= WX) {
        wx -= WX;
        ++wy;
      }
    }
  }
}

// One simulation: one CTA per tile.
template <bool PUSH, bool MOVE, int BC, int TS>
__global__ void SPX_SLOT_BOUNDS(TS) k_slot(const __grid_constant__ StepArgs a) {
  extern __shared__ float smem[];
  // gridDim.y > 1: CTA (tile, s) handles species s of the tile only
  const int s0 = gridDim.y > 1 ? (int)blockIdx.y : 0, s1 = gridDim.y > 1 ? s0 + 1 : a.ns;
  slot_tile<PUSH, MOVE, false, BC, TS>(a, blockIdx.x, smem, s0, s1);
}

// Compensated current sums: the extra registers allow one 256-thread CTA per SM.
template <bool PUSH, int BC>
__global__ void __launch_bounds__(256, 1) k_slot_comp(const __grid_constant__ StepArgs a) {
  extern __shared__ float smem[];
  const int s0 = gridDim.y > 1 ? (int)blockIdx.y : 0, s1 = gridDim.y > 1 ? s0 + 1 : a.ns;
  slot_tile<PUSH, true, true, BC>(a, blockIdx.x, smem, s0, s1);
}

// the instantiation for (push, move, compensated, boundaries, tile shape)
template <int BC, int TS>
static void launch_slot(bool push, bool move, bool comp, dim3 grid, int threads, size_t smem, cudaStream_t st,
                        const StepArgs& a) {
  if (comp && push)
    k_slot_comp<true, BC><<<grid, threads, smem, st>>>(a);
  else if (comp)
    k_slot_comp<false, BC><<<grid, threads, smem, st>>>(a);
  else if (push && move)
    k_slot<true, true, BC, TS><<<grid, threads, smem, st>>>(a);
  else if (push)
    k_slot<true, false, BC, TS><<<grid, threads, smem, st>>>(a);
  else if (move)
    k_slot<false, true, BC, TS><<<grid, threads, smem, st>>>(a);
}

// Many simulations: persistent CTAs take (simulation, tile) items from a work
// queue (an atomic counter over a list sorted by decreasing work), so uneven
// grids and particle counts share one launch and balance across the SMs.
template <bool PUSH, bool MOVE, int BC, int TS>
__global__ void SPX_SLOT_BOUNDS(TS)
    k_slot_batch(const StepArgs* __restrict__ args, const int2* __restrict__ items, int nitems, int* counter) {
  extern __shared__ float smem[];
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const int2 item = items[it];
    slot_tile<PUSH, MOVE, false, BC, TS>(args[item.x], item.y, smem, 0, args[item.x].ns);
    __syncthreads();  // the shared windows are reused by the next item
  }
}

// Overflow fallback: particles parked in the overflow list (no free slot in
// their cell) get the same per-particle work with global gathers and global
// atomic deposits.
template <bool PUSH, bool MOVE>
__device__ __forceinline__ void slot_overflow(const StepArgs& a, int s);

template <bool PUSH, bool MOVE>
__global__ void k_slot_overflow(const __grid_constant__ StepArgs a, int s) {
  slot_overflow<PUSH, MOVE>(a, s);
}

// batch form: blockIdx.y = simulation, every species of it
template <bool PUSH, bool MOVE>
__global__ void k_slot_overflow_batch(const StepArgs* __restrict__ args) {
  const StepArgs& a = args[blockIdx.y];
  for (int s = 0; s < a.ns; ++s) slot_overflow<PUSH, MOVE>(a, s);
}

template <bool PUSH, bool MOVE>
__device__ __forceinline__ void slot_overflow(const StepArgs& a, int s) {
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
      float gth[6];
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const float* src = f == 0 ? a.f.E[0] : f == 1 ? a.f.E[1] : f == 2 ? a.f.E[2] : f == 3 ? a.f.B[0]
                           : f == 4 ? a.f.B[1] : a.f.B[2];
        const float* b = src + (size_t)(iy - 1) * W + (ix - 1);
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
      S.ropx[i] = px;
      S.ropy[i] = py;
      S.ropz[i] = pz;
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

// batch: clear the overflow lists the coming step writes, and the work-queue counter
__global__ void k_batch_reset(const StepArgs* __restrict__ args, int nsims, int* counter) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *counter = 0;
  if (i < nsims)
    for (int s = 0; s < args[i].ns; ++s) *args[i].sp[s].wocount = 0;
}

static SpeciesArgs species_args(Species& sp) {
  SlotSpecies& s = sp.slot;
  const int r = s.ocur, w = s.ocur ^ 1;
  SpeciesArgs A;
  A.dx = s.dx;
  A.dy = s.dy;
  A.px = s.px;
  A.py = s.py;
  A.pz = s.pz;
  A.tag = s.tag;
  A.nlow = s.nlow;
  A.ain = s.narr + (size_t)r * s.ncells;
  A.aout = s.narr + (size_t)w * s.ncells;
  A.rocell = s.ocell[r];
  A.rodx = s.odx[r];
  A.rody = s.ody[r];
  A.ropx = s.opx[r];
  A.ropy = s.opy[r];
  A.ropz = s.opz[r];
  A.rotag = s.otag[r];
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
  A.KL = s.KL;
  A.H = s.H;
  A.rin = s.KL + r * s.H;
  A.rout = s.KL + w * s.H;
  return A;
}

template <int BC, int TS>
static void set_batch_attributes() {
  for (const void* f : {(const void*)k_slot_batch<true, true, BC, TS>, (const void*)k_slot_batch<true, false, BC, TS>,
                        (const void*)k_slot_batch<false, true, BC, TS>})
    SPX_CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
}
template <int BC, int TS>
static void set_single_attributes() {
  for (const void* f : {(const void*)k_slot<true, true, BC, TS>, (const void*)k_slot<true, false, BC, TS>,
                        (const void*)k_slot<false, true, BC, TS>, (const void*)k_slot_comp<true, BC>,
                        (const void*)k_slot_comp<false, BC>})
    SPX_CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
}

template <int TS>
static void set_attributes() {
  set_single_attributes<BC_PERIODIC, TS>();
  set_single_attributes<BC_WALL, TS>();
  set_batch_attributes<BC_ANY, TS>();
  set_batch_attributes<BC_PERIODIC, TS>();
  set_batch_attributes<BC_WALL, TS>();
}
void slot_set_kernel_attributes() {
  set_attributes<0>();
  set_attributes<8>();
  set_attributes<16>();
  set_attributes<168>();
}

// compile-time tile code of a tile shape: 16 (16x16), 8 (8x8), 168 (16x8) or 0 (any other shape)
static int tile_side(const ParticleGeom& pg) {
  return pg.TX == 16 && pg.TY == 16 ? 16 : pg.TX == 8 && pg.TY == 8 ? 8 : pg.TX == 16 && pg.TY == 8 ? 168 : 0;
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
    if (move) SPX_CUDA_TRY(cudaMemsetAsync(sp[s].slot.ocount + (sp[s].slot.ocur ^ 1), 0, sizeof(uint32_t), st));
  }
  const int TC = pg.TC();
  const bool comp = pp.compensated && move;
  const size_t smem = slot_smem_floats(pg.TX, pg.TY, push, move, comp) * sizeof(float);
  const int ts = tile_side(pg);
  // a grid whose tiles fill less than one wave of CTAs (148 SMs x 512 threads)
  // takes one CTA per (tile, species): the species' particles are independent and
  // the CTAs' deposit windows are added into the fields with atomics anyway
  const bool split = a.ns > 1 && (size_t)pg.ntiles() * TC < (size_t)148 * 512;
  const dim3 grid(pg.ntiles(), split ? a.ns : 1);
  if (pp.periodic_x)
    ts == 16    ? launch_slot<BC_PERIODIC, 16>(push, move, comp, grid, TC, smem, st, a)
    : ts == 8   ? launch_slot<BC_PERIODIC, 8>(push, move, comp, grid, TC, smem, st, a)
    : ts == 168 ? launch_slot<BC_PERIODIC, 168>(push, move, comp, grid, TC, smem, st, a)
                : launch_slot<BC_PERIODIC, 0>(push, move, comp, grid, TC, smem, st, a);
  else
    ts == 16    ? launch_slot<BC_WALL, 16>(push, move, comp, grid, TC, smem, st, a)
    : ts == 8   ? launch_slot<BC_WALL, 8>(push, move, comp, grid, TC, smem, st, a)
    : ts == 168 ? launch_slot<BC_WALL, 168>(push, move, comp, grid, TC, smem, st, a)
                : launch_slot<BC_WALL, 0>(push, move, comp, grid, TC, smem, st, a);
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
  if (move)
    for (int s = s0; s < s1; ++s) sp[s].slot.ocur ^= 1;
  SPX_CUDA_TRY(cudaGetLastError());
  return launches;
}

// ---------------------------------------------------------------- batches of simulations
void SlotBatch::release() {
  for (auto& p : d_args)
    if (p) cudaFree(p), p = nullptr;
  if (d_items) cudaFree(d_items);
  if (d_counter) cudaFree(d_counter);
  d_items = nullptr;
  d_counter = nullptr;
  nitems = 0;
}

void slot_batch_build(SlotBatch& b, const std::vector<SlotBatchSim>& sims) {
  b.release();
  b.nsims = (int)sims.size();
  // work items, heaviest tiles first (particles of the simulation per tile)
  std::vector<std::pair<double, int2>> w;
  for (int i = 0; i < b.nsims; ++i) {
    const SlotBatchSim& m = sims[i];
    double per_tile = 0;
    for (int s = 0; s < m.ns; ++s) per_tile += (double)m.sp[s].n / m.pg.ntiles();
    for (int t = 0; t < m.pg.ntiles(); ++t) w.push_back({per_tile, make_int2(i, t)});
  }
  std::stable_sort(w.begin(), w.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  std::vector<int2> items;
  for (auto& x : w) items.push_back(x.second);
  b.nitems = (int)items.size();
  SPX_CUDA_TRY(cudaMalloc(&b.d_items, items.size() * sizeof(int2)));
  SPX_CUDA_TRY(cudaMemcpy(b.d_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
  SPX_CUDA_TRY(cudaMalloc(&b.d_counter, sizeof(int)));
  // argument tables for the two overflow-list parities (all species advance together)
  for (int par = 0; par < 2; ++par) {
    std::vector<StepArgs> h(b.nsims);
    for (int i = 0; i < b.nsims; ++i) {
      const SlotBatchSim& m = sims[i];
      StepArgs& a = h[i];
      a.ns = m.ns;
      a.f = m.fp;
      a.g = m.pg.g;
      a.TX = m.pg.TX;
      a.TY = m.pg.TY;
      a.logTX = m.pg.logTX;
      a.logTY = m.pg.logTY;
      a.NTX = m.pg.NTX;
      a.p = m.pp;
      a.derr = m.derr;
      for (int s = 0; s < m.ns; ++s) {
        Species sp = m.sp[s];
        sp.slot.ocur = par;
        a.sp[s] = species_args(sp);
      }
    }
    SPX_CUDA_TRY(cudaMalloc(&b.d_args[par], h.size() * sizeof(StepArgs)));
    SPX_CUDA_TRY(cudaMemcpy(b.d_args[par], h.data(), h.size() * sizeof(StepArgs), cudaMemcpyHostToDevice));
  }
  const size_t smem = slot_smem_floats(sims[0].pg.TX, sims[0].pg.TY, true, true) * sizeof(float);
  // resident CTAs of the instantiation the steps launch (its register budget depends on the tile shape)
  const int ts = tile_side(sims[0].pg);
  const void* kern = ts == 16    ? (const void*)k_slot_batch<true, true, BC_ANY, 16>
                     : ts == 8   ? (const void*)k_slot_batch<true, true, BC_ANY, 8>
                     : ts == 168 ? (const void*)k_slot_batch<true, true, BC_ANY, 168>
                                 : (const void*)k_slot_batch<true, true, BC_ANY, 0>;
  int per_sm = 0;
  SPX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, sims[0].pg.TC(), smem));
  int dev = 0, nsm = 0;
  SPX_CUDA_TRY(cudaGetDevice(&dev));
  SPX_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  b.grid = std::max(1, std::min(b.nitems, std::max(per_sm, 1) * nsm));
}

template <int BC, int TS>
static void launch_batch(bool push, bool move, const SlotBatch& b, int TC, size_t smem, cudaStream_t st,
                         const StepArgs* args) {
  if (push && move)
    k_slot_batch<true, true, BC, TS><<<b.grid, TC, smem, st>>>(args, b.d_items, b.nitems, b.d_counter);
  else if (push)
    k_slot_batch<true, false, BC, TS><<<b.grid, TC, smem, st>>>(args, b.d_items, b.nitems, b.d_counter);
  else
    k_slot_batch<false, true, BC, TS><<<b.grid, TC, smem, st>>>(args, b.d_items, b.nitems, b.d_counter);
}

int slot_batch_step(SlotBatch& b, std::vector<SlotBatchSim>& sims, bool push, bool move, cudaStream_t st) {
  const int par = sims[0].sp[0].slot.ocur;
  const StepArgs* args = b.d_args[par];
  const int TC = sims[0].pg.TC();
  const size_t smem = slot_smem_floats(sims[0].pg.TX, sims[0].pg.TY, push, move) * sizeof(float);
  int launches = 0;
  k_batch_reset<<<(b.nsims + 255) / 256, 256, 0, st>>>(args, b.nsims, b.d_counter);
  ++launches;
  const int ts = tile_side(sims[0].pg);  // one tile shape for the whole batch
  bool all_periodic = true, all_wall = true;
  for (auto& m : sims) {
    all_periodic = all_periodic && m.pp.periodic_x;
    all_wall = all_wall && !m.pp.periodic_x;
  }
  const int bc = all_periodic ? BC_PERIODIC : all_wall ? BC_WALL : BC_ANY;
#define SPX_BATCH(BCV)                                                       \
  (ts == 16    ? launch_batch<BCV, 16>(push, move, b, TC, smem, st, args)    \
   : ts == 8   ? launch_batch<BCV, 8>(push, move, b, TC, smem, st, args)     \
   : ts == 168 ? launch_batch<BCV, 168>(push, move, b, TC, smem, st, args)   \
               : launch_batch<BCV, 0>(push, move, b, TC, smem, st, args))
  if (bc == BC_PERIODIC)
    SPX_BATCH(BC_PERIODIC);
  else if (bc == BC_WALL)
    SPX_BATCH(BC_WALL);
  else
    SPX_BATCH(BC_ANY);
#undef SPX_BATCH
  ++launches;
  const dim3 og(16, b.nsims);
  if (push && move)
    k_slot_overflow_batch<true, true><<<og, 256, 0, st>>>(args);
  else if (push)
    k_slot_overflow_batch<true, false><<<og, 256, 0, st>>>(args);
  else
    k_slot_overflow_batch<false, true><<<og, 256, 0, st>>>(args);
  ++launches;
  if (move)
    for (auto& m : sims)
      for (int s = 0; s < m.ns; ++s) m.sp[s].slot.ocur ^= 1;
  SPX_CUDA_TRY(cudaGetLastError());
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

__global__ void k_scatter(uint64_t n, uint32_t tag0, const uint32_t* cell, const float* dx, const float* dy,
                          const float* px, const float* py, const float* pz, const uint32_t* tag, uint32_t* cursor,
                          float* odx,
                          float* ody, float* opx, float* opy, float* opz, uint32_t* otag, int K, int TX, int TY,
                          int logTX, int logTY, int NTX) {
  const int TC = TX * TY;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const size_t gc = cell_gc(cell[i], TX, TY, logTX, logTY, NTX);
    const uint32_t r = atomicAdd(&cursor[gc], 1u);
    if ((int)r >= K) continue;  // cannot happen: the low range holds the largest count
    const size_t tile = gc / TC, c = gc - tile * TC;
    const size_t o = tile * (size_t)K * TC + (size_t)r * TC + c;
    odx[o] = dx[i];
    ody[o] = dy[i];
    opx[o] = px[i];
    opy[o] = py[i];
    opz[o] = pz[i];
    otag[o] = tag ? tag[i] : tag0 + (uint32_t)i;
  }
}

void slot_count(const ParticleGeom& pg, uint64_t n, const uint32_t* cell, uint32_t* counts, cudaStream_t st,
                bool reset) {
  if (reset) SPX_CUDA_TRY(cudaMemsetAsync(counts, 0, pg.ncells() * sizeof(uint32_t), st));
  if (n) k_count<<<148 * 8, 256, 0, st>>>(n, cell, counts, pg.TX, pg.TY, pg.logTX, pg.logTY, pg.NTX);
  SPX_CUDA_TRY(cudaGetLastError());
}

void slot_scatter_begin(Species& s, const ParticleGeom& pg, uint32_t* cursor, cudaStream_t st) {
  s.slot.ocur = 0;
  SPX_CUDA_TRY(cudaMemsetAsync(cursor, 0, pg.ncells() * sizeof(uint32_t), st));
}

void slot_scatter_chunk(Species& s, const ParticleGeom& pg, uint64_t n, uint32_t tag0, const uint32_t* cell,
                        const float* dx, const float* dy, const float* px, const float* py, const float* pz,
                        const uint32_t* tag, uint32_t* cursor, cudaStream_t st) {
  SlotSpecies& S = s.slot;
  if (n)
    k_scatter<<<148 * 8, 256, 0, st>>>(n, tag0, cell, dx, dy, px, py, pz, tag, cursor, S.dx, S.dy, S.px, S.py, S.pz,
                                       S.tag, S.K, pg.TX, pg.TY, pg.logTX, pg.logTY, pg.NTX);
  SPX_CUDA_TRY(cudaGetLastError());
}

void slot_scatter_end(Species& s, const ParticleGeom& pg, uint32_t* cursor, cudaStream_t st) {
  SlotSpecies& S = s.slot;
  SPX_CUDA_TRY(cudaMemcpyAsync(S.nlow, cursor, pg.ncells() * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  SPX_CUDA_TRY(cudaMemsetAsync(S.narr, 0, 2 * pg.ncells() * sizeof(uint32_t), st));
  SPX_CUDA_TRY(cudaMemsetAsync(S.ocount, 0, 2 * sizeof(uint32_t), st));
  SPX_CUDA_TRY(cudaGetLastError());
}

void slot_scatter(Species& s, const ParticleGeom& pg, uint64_t n, const uint32_t* cell, const float* dx,
                  const float* dy, const float* px, const float* py, const float* pz, const uint32_t* tag,
                  uint32_t* cursor, cudaStream_t st) {
  slot_scatter_begin(s, pg, cursor, st);
  slot_scatter_chunk(s, pg, n, 0u, cell, dx, dy, px, py, pz, tag, cursor, st);
  slot_scatter_end(s, pg, cursor, st);
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
    const int nlow = (int)S.nlow[gc], nin = (int)S.ain[gc];
    const size_t base = tile * (size_t)S.K * TC + c;
    for (int n = 0; n < nlow + nin; ++n) {
      const int slot = n < nlow ? n : S.rin + (n - nlow);
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

__global__ void k_max_occ(const uint32_t* nlow, const uint32_t* ain, size_t n, uint32_t* out) {
  uint32_t m = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = max(m, nlow[i] + (ain ? ain[i] : 0u));
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

void slot_max_occupancy(const Species& s, const ParticleGeom& pg, uint32_t* d_out, cudaStream_t st) {
  const SlotSpecies& S = s.slot;
  k_max_occ<<<148 * 4, 256, 0, st>>>(S.nlow, S.narr ? S.narr + (size_t)S.ocur * pg.ncells() : nullptr, pg.ncells(),
                                     d_out);
  SPX_CUDA_TRY(cudaGetLastError());
}

void slot_allocate(Species& s, const ParticleGeom& pg, int KL, int H, uint64_t n) {
  SlotSpecies& S = s.slot;
  const int K = KL + 2 * H;
  const size_t cap = pg.ncells() * (size_t)K;
  S.K = K;
  S.KL = KL;
  S.H = H;
  S.ncells = pg.ncells();
  S.ocap = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(1u << 16, n / 32), 1u << 28);
  // one allocation carved into the slot arrays, the counters and both overflow lists
  // (one cudaMalloc per species instead of 23: a batch of many small simulations sets up
  // hundreds of species)
  const auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t slots = up(cap * 4), cells = up(pg.ncells() * 4), ovf = up((size_t)S.ocap * 4);
  const size_t total = 6 * slots + 3 * cells + 14 * ovf + 256;
  SPX_CUDA_TRY(cudaMalloc(&S.block, total));
  char* p = static_cast<char*>(S.block);
  auto take = [&](size_t b) {
    char* q = p;
    p += b;
    return q;
  };
  S.dx = reinterpret_cast<float*>(take(slots));
  S.dy = reinterpret_cast<float*>(take(slots));
  S.px = reinterpret_cast<float*>(take(slots));
  S.py = reinterpret_cast<float*>(take(slots));
  S.pz = reinterpret_cast<float*>(take(slots));
  S.tag = reinterpret_cast<uint32_t*>(take(slots));
  // nlow, narr and ocount are set by slot_scatter_end, on the stream of the scatter
  S.nlow = reinterpret_cast<uint32_t*>(take(cells));
  S.narr = reinterpret_cast<uint32_t*>(take(2 * cells));
  for (int b = 0; b < 2; ++b) {
    S.ocell[b] = reinterpret_cast<uint32_t*>(take(ovf));
    S.odx[b] = reinterpret_cast<float*>(take(ovf));
    S.ody[b] = reinterpret_cast<float*>(take(ovf));
    S.opx[b] = reinterpret_cast<float*>(take(ovf));
    S.opy[b] = reinterpret_cast<float*>(take(ovf));
    S.opz[b] = reinterpret_cast<float*>(take(ovf));
    S.otag[b] = reinterpret_cast<uint32_t*>(take(ovf));
  }
  S.ocount = reinterpret_cast<uint32_t*>(take(256));
}

void slot_release(Species& s) {
  SlotSpecies& S = s.slot;
  if (S.block) cudaFree(S.block);
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

// ---------------------------------------------------------------- tracked particles
// save/mod.rs:94-96 in FP32: (ix as Float + dx) / c, (iy as Float + dy) / c, psa
__device__ __forceinline__ void put_tracked(int32_t r, uint32_t cx, uint32_t cy, float dx, float dy, float px,
                                            float py, float pz, float c, float csqinv, float* x, float* y, float* g) {
  x[r] = ((float)cx + dx) / c;
  y[r] = ((float)cy + dy) / c;
  g[r] = gamma_of(px, py, pz, csqinv);
}

__global__ void k_tracked_slot(SpeciesArgs S, int TX, int TY, int logTX, int NTX, size_t ncells, const int32_t* rank,
                               float c, float csqinv, float* x, float* y, float* g) {
  const int TC = TX * TY;
  for (size_t gc = blockIdx.x * (size_t)blockDim.x + threadIdx.x; gc < ncells; gc += (size_t)gridDim.x * blockDim.x) {
    const size_t tile = gc / TC;
    const int cc = (int)(gc - tile * TC);
    const uint32_t cx = (uint32_t)((tile % NTX) * TX + (cc & (TX - 1)) + 1);
    const uint32_t cy = (uint32_t)((tile / NTX) * TY + (cc >> logTX) + 1);
    const int nlow = (int)S.nlow[gc], nin = (int)S.ain[gc];
    const size_t base = tile * (size_t)S.K * TC + cc;
    for (int n = 0; n < nlow + nin; ++n) {
      const size_t i = base + (size_t)(n < nlow ? n : S.rin + (n - nlow)) * TC;
      const int32_t r = rank[S.tag[i]];
      if (r >= 0) put_tracked(r, cx, cy, S.dx[i], S.dy[i], S.px[i], S.py[i], S.pz[i], c, csqinv, x, y, g);
    }
  }
}

__global__ void k_tracked_overflow(SpeciesArgs S, const int32_t* rank, float c, float csqinv, float* x, float* y,
                                   float* g) {
  const uint32_t n = min(*S.rocount, S.ocap);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int32_t r = rank[S.rotag[i]];
    if (r >= 0)
      put_tracked(r, S.rocell[i] & 0xFFFFu, S.rocell[i] >> 16, S.rodx[i], S.rody[i], S.ropx[i], S.ropy[i], S.ropz[i],
                  c, csqinv, x, y, g);
  }
}

__global__ void k_tracked_plain(PlainSpecies P, uint64_t n, const int32_t* rank, float c, float csqinv, float* x,
                                float* y, float* g) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t r = rank[i];
    if (r < 0) continue;
    const int cx = (int)floorf(P.x[i] + 0.5f), cy = (int)floorf(P.y[i] + 0.5f);
    put_tracked(r, (uint32_t)cx, (uint32_t)cy, P.x[i] - (float)cx, P.y[i] - (float)cy, P.px[i], P.py[i], P.pz[i], c,
                csqinv, x, y, g);
  }
}

void gather_tracked(const Species& s, const ParticleGeom& pg, bool plain, const int32_t* rank, float c, float* x,
                    float* y, float* g, cudaStream_t st) {
  const float csqinv = 1.0f / (c * c);
  if (plain) {
    if (s.n) k_tracked_plain<<<148 * 4, 256, 0, st>>>(s.plain, s.n, rank, c, csqinv, x, y, g);
  } else {
    SpeciesArgs A = species_args(const_cast<Species&>(s));
    k_tracked_slot<<<148 * 4, 256, 0, st>>>(A, pg.TX, pg.TY, pg.logTX, pg.NTX, pg.ncells(), rank, c, csqinv, x, y, g);
    k_tracked_overflow<<<16, 256, 0, st>>>(A, rank, c, csqinv, x, y, g);
  }
  SPX_CUDA_TRY(cudaGetLastError());
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
    const int nlow = (int)S.nlow[gc], nin = (int)S.ain[gc];
    const size_t base = tile * (size_t)S.K * TC + cc;
    for (int n = 0; n < nlow + nin; ++n) {
      const int slot = n < nlow ? n : S.rin + (n - nlow);
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

__global__ void k_init(InitSpec is, int ny, uint64_t off, uint64_t n, uint32_t* cell, float* dxo, float* dyo,
                       float* pxo, float* pyo, float* pzo) {
  const int ncols = is.x1 - is.x0;
  const float c = is.c;
  const float csqinv = 1.0f / (c * c);
  const float g = is.gamma_drift;
  const float beta_inj = g > 1.0f ? is.sign_x * sqrtf(1.0f - 1.0f / (g * g)) : 0.0f;  // src/prtls.rs:224
  for (uint64_t o = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; o < n; o += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = off + o;  // particle index in the species (its RNG counter)
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
    cell[o] = (uint32_t)ix | ((uint32_t)iy << 16);
    dxo[o] = dx;
    dyo[o] = dy;
    pxo[o] = px;
    pyo[o] = py;
    pzo[o] = pz;
  }
}

void init_particles(const InitSpec& is, const Grid& g, uint64_t off, uint64_t n, uint32_t* cell, float* dx,
                    float* dy, float* px, float* py, float* pz, cudaStream_t st) {
  if (n) k_init<<<148 * 16, 256, 0, st>>>(is, g.ny, off, n, cell, dx, dy, px, py, pz);
  SPX_CUDA_TRY(cudaGetLastError());
}

}  // namespace spx
