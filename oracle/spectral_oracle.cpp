// CPU oracle for the spectral_rs per-timestep hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++, the algorithm of
// the reference Rust crate (pcrumley/spectral_rs) for particle push, position
// update, boundary conditions, current/density deposition and the
// pseudo-spectral field update.  It is the checker the GPU library is compared
// against and the CPU baseline that bench.py times; the product path
// (libspectral_gpu.so) never links or calls it.
//
// It is templated on the reference's `Float` alias (src/lib.rs:15-19):
//   float  = the reference FP32 path (default build),
//   double = the reference `--features dprec` build (used as the FP64 oracle).
//
// Arithmetic order follows the reference line for line.  Build with
// -ffp-contract=off and no fast-math: rustc never fuses a*b+c, `x.powi(-1)` is
// the correctly rounded 1/x, and `sqrt` is IEEE.  Complex arithmetic restates
// num_complex's component formulas (not std::complex, whose operator* may
// take C99 Annex G paths).
//
// The one deliberate deviation: the FFT.  The reference calls the third-party
// crate `rustfft` (Cargo.toml:22, "6.0.0" caret range, no Cargo.lock, so the
// resolved version is unpinned).  Its published algorithm is an unnormalized
// DFT X[k] = sum_n x[n] exp(-2*pi*i*k*n/N) (forward) and exp(+...) (inverse),
// numpy's convention; rustfft's own f32 rounding is not reproducible here.  The
// oracle evaluates each 1-D transform in double precision (iterative radix-2
// for powers of two, a direct DFT otherwise) and rounds the result to Float
// after each 1-D pass, exactly where the reference stores Float between its
// row and column passes (src/flds/fft_2d.rs:91-172).  It is pinned against the
// reference's numpy-generated golden vectors (fft_2d.rs:478-547, 601-907).
//
// CPU parallelism mirrors the reference: the deposition, position update and
// boundary passes are serial (src/lib.rs:266-489, src/prtls.rs:86-190); the
// Boris push runs in parallel chunks of PRTL_CHUNK_SIZE=1000 particles
// (src/prtls.rs:288-300, src/lib.rs:23); the filter stencil and FFT rows are
// parallel (src/flds/field.rs:385-420, fft_2d.rs:97-127).  OpenMP stands in
// for rayon.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const size_t PRTL_CHUNK_SIZE = 1000;  // src/lib.rs:23

// ---------------------------------------------------------------- complex
// num_complex::Complex<T> arithmetic, component by component.
template <typename T>
struct Cx {
  T re, im;
};
template <typename T>
static inline Cx<T> cmul(Cx<T> a, Cx<T> b) {  // impl Mul for Complex
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
static inline Cx<T> cscale(Cx<T> a, T s) {  // Complex * T   and   T * Complex
  return {a.re * s, a.im * s};
}
template <typename T>
static inline Cx<T> sscale(T s, Cx<T> a) {  // T * Complex (num_complex: self * re, self * im)
  return {s * a.re, s * a.im};
}
template <typename T>
static inline Cx<T> cadd(Cx<T> a, Cx<T> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename T>
static inline Cx<T> csub(Cx<T> a, Cx<T> b) {
  return {a.re - b.re, a.im - b.im};
}

// ---------------------------------------------------------------- params
template <typename T>
struct Sim {  // src/lib.rs:204-217 (the fields the hot path reads)
  size_t size_x, size_y, delta;
  T dt, c;
  uint32_t dens;
  T gamma_inj;
  uint32_t n_pass;
  bool periodic_x;  // cargo feature `periodic` (src/prtls.rs:136)
  bool left_wall;   // additive: mirror of the right wall at ix = delta + 1 (off = reference)
};

// ---------------------------------------------------------------- Field
// src/flds/field.rs:17-23.  spatial: (ny+2)x(nx+2) row-major with a one-cell
// ghost frame; spectral: ny x nx complex.
template <typename T>
struct Field {
  size_t nx = 0, ny = 0;
  std::vector<T> spatial;
  std::vector<Cx<T>> spectral;
  void init(size_t nx_, size_t ny_) {
    nx = nx_;
    ny = ny_;
    spatial.assign((ny + 2) * (nx + 2), T(0));
    spectral.assign(ny * nx, Cx<T>{T(0), T(0)});
  }
};

// field.rs:78-107
template <typename T>
static void copy_to_spectral(Field<T>& f) {
  for (size_t iy = 0; iy < f.ny; ++iy) {
    size_t ij = iy * f.nx;
    size_t ijg = (iy + 1) * (f.nx + 2);
    for (size_t ix = 0; ix < f.nx; ++ix) {
      f.spectral[ij + ix].re = f.spatial[ijg + ix + 1];
      f.spectral[ij + ix].im = T(0);
    }
  }
}

// field.rs:142-257: periodic fill of the ghost frame.
template <typename T>
static void update_ghosts(std::vector<T>& fld, size_t nx, size_t ny) {
  const size_t W = nx + 2;
  for (size_t i = 0; i < nx; ++i) fld[0 * W + 1 + i] = fld[ny * W + 1 + i];          // top ghost <- last row
  for (size_t i = 0; i < nx; ++i) fld[(ny + 1) * W + 1 + i] = fld[1 * W + 1 + i];    // bottom ghost <- first row
  for (size_t r = 1; r <= ny; ++r) fld[r * W + 0] = fld[r * W + nx];                 // left ghost <- last col
  for (size_t r = 1; r <= ny; ++r) fld[r * W + nx + 1] = fld[r * W + 1];             // right ghost <- first col
  fld[0] = fld[ny * W + nx];                     // top-left     <- bottom-right
  fld[nx + 1] = fld[ny * W + 1];                 // top-right    <- bottom-left
  fld[(ny + 1) * W + 0] = fld[1 * W + nx];       // bottom-left  <- top-right
  fld[(ny + 1) * W + nx + 1] = fld[1 * W + 1];   // bottom-right <- top-left
}

// field.rs:110-139
template <typename T>
static void copy_to_spatial(Field<T>& f) {
  for (size_t iy = 0; iy < f.ny; ++iy) {
    size_t ij = iy * f.nx;
    size_t ijg = (iy + 1) * (f.nx + 2);
    for (size_t ix = 0; ix < f.nx; ++ix) f.spatial[ijg + ix + 1] = f.spectral[ij + ix].re;
  }
  update_ghosts(f.spatial, f.nx, f.ny);
}

// field.rs:260-373: fold the ghost frame onto the opposite interior edge.
// The ghost cells keep their values (the reference never clears them).
template <typename T>
static void deposit_ghosts(std::vector<T>& fld, size_t nx, size_t ny) {
  const size_t W = nx + 2;
  for (size_t i = 0; i < nx; ++i) fld[ny * W + 1 + i] += fld[0 * W + 1 + i];
  for (size_t i = 0; i < nx; ++i) fld[1 * W + 1 + i] += fld[(ny + 1) * W + 1 + i];
  for (size_t r = 1; r <= ny; ++r) fld[r * W + nx] += fld[r * W + 0];
  for (size_t r = 1; r <= ny; ++r) fld[r * W + 1] += fld[r * W + nx + 1];
  fld[ny * W + nx] += fld[0];
  fld[ny * W + 1] += fld[nx + 1];
  fld[1 * W + nx] += fld[(ny + 1) * W + 0];
  fld[1 * W + 1] += fld[(ny + 1) * W + nx + 1];
}

// field.rs:376-426.  The reference also evaluates the stencil on the bottom
// ghost row, reading one row past the end of the array (undefined behaviour);
// update_ghosts then overwrites that row, so only rows 1..ny are computed here.
template <typename T>
static void binomial_filter_2_d(std::vector<T>& fld, std::vector<T>& wrk, size_t nx, size_t ny) {
  const size_t W = nx + 2;
  const T* in = fld.data();
  T* out = wrk.data();
#pragma omp parallel for schedule(static)
  for (long r = 1; r <= (long)ny; ++r) {
    for (size_t col = 1; col <= nx; ++col) {
      size_t i = (size_t)r * W + col;
      size_t ijm1 = i - 2 - nx;
      size_t ijp1 = i + 2 + nx;
      T v = T(0.0625) * in[ijm1 - 1];
      v += T(0.125) * in[ijm1];
      v += T(0.0625) * in[ijm1 + 1];
      v += T(0.125) * in[i - 1];
      v += T(0.25) * in[i];
      v += T(0.125) * in[i + 1];
      v += T(0.0625) * in[ijp1 - 1];
      v += T(0.125) * in[ijp1];
      v += T(0.0625) * in[ijp1 + 1];
      out[i] = v;
    }
  }
  update_ghosts(wrk, nx, ny);
  fld = wrk;  // the serial copy-back (field.rs:423-425); wrk's frame is now periodic
}

// ---------------------------------------------------------------- FFT
// One unnormalized 1-D DFT in double precision.  sign=-1 forward, +1 inverse.
struct Plan1D {
  size_t n = 0;
  bool pow2 = false;
  std::vector<double> cs, sn;  // exp(-2 pi i k / n) = cs[k] - i sn[k]... stored as cos, sin
  void init(size_t n_) {
    n = n_;
    pow2 = n && !(n & (n - 1));
    cs.resize(n);
    sn.resize(n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (size_t k = 0; k < n; ++k) {
      long double a = two_pi * (long double)k / (long double)n;
      cs[k] = (double)cosl(a);
      sn[k] = (double)sinl(a);
    }
  }
  void run(std::vector<double>& re, std::vector<double>& im, int sign) const {
    if (!pow2) {
      std::vector<double> orr(n), oi(n);
      for (size_t k = 0; k < n; ++k) {
        double sr = 0, si = 0;
        for (size_t j = 0; j < n; ++j) {
          size_t m = (k * j) % n;
          double c = cs[m], s = sign * sn[m];  // exp(sign * 2 pi i m/n)
          sr += re[j] * c - im[j] * s;
          si += re[j] * s + im[j] * c;
        }
        orr[k] = sr;
        oi[k] = si;
      }
      re.swap(orr);
      im.swap(oi);
      return;
    }
    // iterative radix-2 decimation in time
    for (size_t i = 1, j = 0; i < n; ++i) {
      size_t bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) {
        std::swap(re[i], re[j]);
        std::swap(im[i], im[j]);
      }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
      size_t step = n / len;
      for (size_t i = 0; i < n; i += len) {
        for (size_t k = 0; k < len / 2; ++k) {
          double wr = cs[k * step], wi = sign * sn[k * step];
          size_t a = i + k, b = i + k + len / 2;
          double tr = re[b] * wr - im[b] * wi;
          double ti = re[b] * wi + im[b] * wr;
          re[b] = re[a] - tr;
          im[b] = im[a] - ti;
          re[a] += tr;
          im[a] += ti;
        }
      }
    }
  }
};

// fft_2d.rs:91-172.  Row transforms of length nx, then column transforms of
// length ny; Float is stored between the passes.  inverse: unnormalized
// inverse, then every entry times (nx*ny as Float).powi(-1).
template <typename T>
static void fft2d(std::vector<Cx<T>>& a, size_t nx, size_t ny, const Plan1D& px, const Plan1D& py,
                  bool inverse) {
  const int sign = inverse ? +1 : -1;
#pragma omp parallel
  {
    std::vector<double> re(nx), im(nx);
#pragma omp for schedule(static)
    for (long r = 0; r < (long)ny; ++r) {
      for (size_t x = 0; x < nx; ++x) {
        re[x] = (double)a[r * nx + x].re;
        im[x] = (double)a[r * nx + x].im;
      }
      px.run(re, im, sign);
      for (size_t x = 0; x < nx; ++x) a[r * nx + x] = {(T)re[x], (T)im[x]};
    }
  }
#pragma omp parallel
  {
    std::vector<double> re(ny), im(ny);
#pragma omp for schedule(static)
    for (long c = 0; c < (long)nx; ++c) {
      for (size_t y = 0; y < ny; ++y) {
        re[y] = (double)a[y * nx + c].re;
        im[y] = (double)a[y * nx + c].im;
      }
      py.run(re, im, sign);
      for (size_t y = 0; y < ny; ++y) a[y * nx + c] = {(T)re[y], (T)im[y]};
    }
  }
  if (inverse) {
    T norm = T(1) / (T)(nx * ny);
    for (auto& v : a) v = cscale(v, norm);  // MulAssign<T>
  }
}

// ---------------------------------------------------------------- wave numbers
// src/flds/wave_num.rs:12-41
template <typename T>
static void wave_numbers(size_t nx, size_t ny, std::vector<T>& kx, std::vector<T>& ky,
                         std::vector<T>& kn) {
  const T PI = (T)3.14159265358979323846;  // std::f64::consts::PI as Float
  kx.assign(nx * ny, T(0));
  ky.assign(nx * ny, T(0));
  kn.assign(nx * ny, T(0));
  for (size_t i = 0; i < ny; ++i) {
    for (size_t j = 0; j < nx; ++j) {
      size_t ind = i * nx + j;
      kx[ind] = (T)j;
      if (j >= nx / 2 + 1) kx[ind] -= (T)nx;
      kx[ind] *= T(2.0) * PI / (T)nx;
      ky[ind] = (T)i;
      if (i >= ny / 2 + 1) ky[ind] -= (T)ny;
      ky[ind] *= T(2.0) * PI / (T)ny;
    }
  }
  for (size_t ind = 1; ind < nx * ny; ++ind) kn[ind] = T(1.0) / (kx[ind] * kx[ind] + ky[ind] * ky[ind]);
}

// ---------------------------------------------------------------- Flds
// src/flds/mod.rs:15-310
template <typename T>
struct Flds {
  Field<T> e_x, e_y, e_z, b_x, b_y, b_z, j_x, j_y, j_z, dens, dsty, wrk;
  std::vector<T> k_x, k_y, k_norm;
  std::vector<Cx<T>> b_x_wrk, b_y_wrk, b_z_wrk;
  Plan1D plan_x, plan_y;
  void init(const Sim<T>& s) {
    for (Field<T>* f : {&e_x, &e_y, &e_z, &b_x, &b_y, &b_z, &j_x, &j_y, &j_z, &dens, &dsty, &wrk})
      f->init(s.size_x, s.size_y);
    wave_numbers(s.size_x, s.size_y, k_x, k_y, k_norm);
    b_x_wrk.assign(s.size_x * s.size_y, Cx<T>{0, 0});
    b_y_wrk = b_x_wrk;
    b_z_wrk = b_x_wrk;
    plan_x.init(s.size_x);
    plan_y.init(s.size_y);
  }
  Field<T>* by_id(int id) {
    // field ids shared with the GPU C ABI (include/spectral_gpu.h)
    switch (id) {
      case 0: return &e_x;
      case 1: return &e_y;
      case 2: return &e_z;
      case 3: return &b_x;
      case 4: return &b_y;
      case 5: return &b_z;
      case 6: return &j_x;
      case 7: return &j_y;
      case 8: return &j_z;
      case 9: return &dsty;
      case 10: return &dens;
      default: return nullptr;
    }
  }

  void update(const Sim<T>& s) {
    const size_t nx = s.size_x, ny = s.size_y, n = nx * ny;
    // mod.rs:90-94 filter currents and charge density
    for (uint32_t p = 0; p < s.n_pass; ++p)
      for (Field<T>* f : {&j_x, &j_y, &j_z, &dsty}) binomial_filter_2_d(f->spatial, wrk.spatial, nx, ny);
    // mod.rs:66-85 copy to spectral, normalise dsty by 1/dens
    for (Field<T>* f : {&j_x, &j_y, &j_z, &e_x, &e_y, &e_z, &dsty}) copy_to_spectral(*f);
    T norm = T(1.0) / (T)s.dens;
    for (auto& v : dsty.spectral) {
      v.re *= norm;
      v.im *= norm;
    }
    // mod.rs:101-103
    for (Field<T>* f : {&j_x, &j_y, &j_z, &dsty}) fft2d(f->spectral, nx, ny, plan_x, plan_y, false);
    // mod.rs:106-108 (j_z[0] is left alone, as in the reference)
    j_x.spectral[0] = {0, 0};
    j_y.spectral[0] = {0, 0};
    // mod.rs:113-119
    b_x.spectral = b_x_wrk;
    b_y.spectral = b_y_wrk;
    b_z.spectral = b_z_wrk;
    // mod.rs:122-124
    for (Field<T>* f : {&e_x, &e_y, &e_z}) fft2d(f->spectral, nx, ny, plan_x, plan_y, false);
    // mod.rs:127-173 Ampere
    const T ckc = s.dt / (T)s.dens;
    const T cdt = s.dt * s.c;
    const Cx<T> icdt{T(0.0), cdt}, micdt{T(0.0), -cdt};
    for (size_t i = 0; i < n; ++i)
      e_x.spectral[i] = cadd(e_x.spectral[i], csub(cmul(cscale(icdt, k_y[i]), b_z.spectral[i]),
                                                   sscale(ckc, j_x.spectral[i])));
    for (size_t i = 0; i < n; ++i)
      e_y.spectral[i] = cadd(e_y.spectral[i], csub(cmul(cscale(micdt, k_x[i]), b_z.spectral[i]),
                                                   sscale(ckc, j_y.spectral[i])));
    for (size_t i = 0; i < n; ++i) {
      Cx<T> kb = csub(sscale(k_x[i], b_y.spectral[i]), sscale(k_y[i], b_x.spectral[i]));
      e_z.spectral[i] = cadd(e_z.spectral[i], cmul(icdt, kb));
      e_z.spectral[i] = csub(e_z.spectral[i], sscale(ckc, j_z.spectral[i]));
    }
    // mod.rs:177-207 divergence ("Boris") correction, k=0 kept
    Cx<T> ex0 = e_x.spectral[0], ey0 = e_y.spectral[0];
    const Cx<T> I{T(0.0), T(1.0)};
    for (size_t i = 0; i < n; ++i) {
      Cx<T> t = cadd(cadd(sscale(k_x[i], e_x.spectral[i]), sscale(k_y[i], e_y.spectral[i])),
                     cmul(I, dsty.spectral[i]));
      t = cscale(t, k_norm[i]);
      e_x.spectral[i] = csub(e_x.spectral[i], cscale(t, k_x[i]));
      e_y.spectral[i] = csub(e_y.spectral[i], cscale(t, k_y[i]));
    }
    e_x.spectral[0] = ex0;
    e_y.spectral[0] = ey0;
    // mod.rs:211-225 Faraday on B at t+1/2
    for (size_t i = 0; i < n; ++i)
      b_x_wrk[i] = csub(b_x_wrk[i], cmul(cscale(icdt, k_y[i]), e_z.spectral[i]));
    for (size_t i = 0; i < n; ++i)
      b_y_wrk[i] = cadd(b_y_wrk[i], cmul(cscale(icdt, k_x[i]), e_z.spectral[i]));
    for (size_t i = 0; i < n; ++i) {
      Cx<T> d = csub(sscale(k_y[i], e_x.spectral[i]), sscale(k_x[i], e_y.spectral[i]));
      b_z_wrk[i] = cadd(b_z_wrk[i], cmul(icdt, d));
    }
    // mod.rs:230-266 Nyquist column kx = nx/2 and row ky = ny/2
    for (std::vector<Cx<T>>* f : {&b_x_wrk, &b_y_wrk, &b_z_wrk, &e_x.spectral, &e_y.spectral, &e_z.spectral}) {
      for (size_t i = nx / 2; i < n; i += nx) (*f)[i] = {0, 0};
      for (size_t i = (ny * nx) / 2; i < (ny * nx) / 2 + nx; ++i) (*f)[i] = {0, 0};
    }
    // mod.rs:270-278 B at integer time
    for (int c = 0; c < 3; ++c) {
      std::vector<Cx<T>>& bm = c == 0 ? b_x.spectral : c == 1 ? b_y.spectral : b_z.spectral;
      const std::vector<Cx<T>>& bp = c == 0 ? b_x_wrk : c == 1 ? b_y_wrk : b_z_wrk;
      for (size_t i = 0; i < n; ++i) bm[i] = sscale(T(0.5), cadd(bm[i], bp[i]));
    }
    // mod.rs:281-307
    for (Field<T>* f : {&b_x, &b_y, &b_z, &e_x, &e_y, &e_z}) {
      fft2d(f->spectral, nx, ny, plan_x, plan_y, true);
      copy_to_spatial(*f);
    }
  }
};

// ---------------------------------------------------------------- Prtl
// src/prtls.rs:8-23 (tag and track are not on the hot path)
template <typename T>
struct Prtl {
  std::vector<uint64_t> ix, iy;
  std::vector<T> dx, dy, px, py, pz, psa;
  T charge, alpha, beta, vth;
};

enum Err { OK = 0, E_ARG = 1, E_BOUNDS = 2, E_WALL = 3 };

// prtls.rs:86-121
template <typename T>
static int update_position(Prtl<T>& p, const Sim<T>& s) {
  const T dt = s.dt;
  const size_t n = p.ix.size();
  for (size_t i = 0; i < n; ++i) {
    if (p.ix[i] == 0 || p.iy[i] == 0) return E_BOUNDS;  // underflow asserts (:98-102)
    T c1 = T(0.5) * dt * (T(1) / p.psa[i]);
    p.dx[i] += c1 * p.px[i];
    if (p.dx[i] >= T(0.5)) {
      p.dx[i] -= T(1.0);
      p.ix[i] += 1;
    } else if (p.dx[i] < T(-0.5)) {
      p.dx[i] += T(1.0);
      p.ix[i] -= 1;
    }
    p.dy[i] += c1 * p.py[i];
    if (p.dy[i] >= T(0.5)) {
      p.dy[i] -= T(1.0);
      p.iy[i] += 1;
    } else if (p.dy[i] < T(-0.5)) {
      p.dy[i] += T(1.0);
      p.iy[i] -= 1;
    }
  }
  return OK;
}

template <typename T>
static inline T rust_signum(T x) {  // f32::signum: +-1 by the sign bit, NaN for NaN
  if (std::isnan(x)) return x;
  return std::copysign(T(1.0), x);
}

// prtls.rs:124-190
template <typename T>
static int apply_bc(Prtl<T>& p, const Sim<T>& s) {
  const size_t n = p.ix.size();
  for (size_t i = 0; i < n; ++i) {
    if (p.iy[i] < 1)
      p.iy[i] += s.size_y;
    else if (p.iy[i] > s.size_y)
      p.iy[i] -= s.size_y;
  }
  if (s.periodic_x) {
    for (size_t i = 0; i < n; ++i) {
      if (p.ix[i] < 1)
        p.ix[i] += s.size_x;
      else if (p.ix[i] > s.size_x)
        p.ix[i] -= s.size_x;
    }
  } else {
    const uint64_t wall_loc = s.size_x + 1 - s.delta;
    const uint64_t lwall = s.delta + 1;
    if (n) {
      uint64_t mx = *std::max_element(p.ix.begin(), p.ix.end());
      uint64_t mn = *std::min_element(p.ix.begin(), p.ix.end());
      // :154-171; with the optional left wall a particle may sit one cell below it
      if (!(mx <= wall_loc + 1) || !(s.left_wall ? mn + 1 > s.delta : mn > s.delta)) return E_WALL;
    }
    for (size_t i = 0; i < n; ++i) {
      if (s.left_wall && p.ix[i] <= lwall) {  // mirror image of the right wall below
        if (p.ix[i] == lwall) {
          T sgn = rust_signum(p.dx[i]);
          if (sgn < T(0)) {
            p.px[i] *= T(-1.0);
            p.dx[i] *= T(-1.0);
          }
        } else {
          p.dx[i] -= T(1.0);
          p.ix[i] += 1;
          p.px[i] *= T(-1.0);
        }
        continue;
      }
      if (p.ix[i] < wall_loc) {
      } else if (p.ix[i] == wall_loc) {
        T sgn = rust_signum(p.dx[i]);
        p.px[i] *= -sgn;
        p.dx[i] *= -sgn;
      } else {
        p.dx[i] += T(1.0);
        p.ix[i] -= 1;
        p.px[i] *= T(-1.0);
      }
    }
  }
  return OK;
}

// Second-order (TSC) weights, src/lib.rs:339-347 (same text in prtls.rs:321-329).
template <typename T>
struct W9 {
  T w00, w01, w02, w10, w11, w12, w20, w21, w22;
};
template <typename T>
static inline W9<T> weights(T dx, T dy) {
  W9<T> w;
  w.w00 = T(0.5) * (T(0.5) - dy) * (T(0.5) - dy) * T(0.5) * (T(0.5) - dx) * (T(0.5) - dx);
  w.w01 = T(0.5) * (T(0.5) - dy) * (T(0.5) - dy) * (T(0.75) - dx * dx);
  w.w02 = T(0.5) * (T(0.5) - dy) * (T(0.5) - dy) * T(0.5) * (T(0.5) + dx) * (T(0.5) + dx);
  w.w10 = (T(0.75) - dy * dy) * T(0.5) * (T(0.5) - dx) * (T(0.5) - dx);
  w.w11 = (T(0.75) - dy * dy) * (T(0.75) - dx * dx);
  w.w12 = (T(0.75) - dy * dy) * T(0.5) * (T(0.5) + dx) * (T(0.5) + dx);
  w.w20 = T(0.5) * (T(0.5) + dy) * (T(0.5) + dy) * T(0.5) * (T(0.5) - dx) * (T(0.5) - dx);
  w.w21 = T(0.5) * (T(0.5) + dy) * (T(0.5) + dy) * (T(0.75) - dx * dx);
  w.w22 = T(0.5) * (T(0.5) + dy) * (T(0.5) + dy) * T(0.5) * (T(0.5) + dx) * (T(0.5) + dx);
  return w;
}

// src/lib.rs:266-393 (serial, particle order)
template <typename T>
static int deposit_current(const Prtl<T>& p, const Sim<T>& s, Flds<T>& f) {
  T* jx = f.j_x.spatial.data();
  T* jy = f.j_y.spatial.data();
  T* jz = f.j_z.spatial.data();
  const size_t len = f.j_x.spatial.size(), W = 2 + s.size_x;
  const size_t n = p.ix.size();
  for (size_t i = 0; i < n; ++i) {
    size_t ix = p.ix[i], iy = p.iy[i];
    if (iy == 0 || ix == 0) return E_BOUNDS;
    size_t ijm1 = (iy - 1) * W, ij = iy * W, ijp1 = (iy + 1) * W;
    if (!(ijp1 + ix + 1 < len)) return E_BOUNDS;
    T psa_inv = T(1) / p.psa[i];
    T vx = p.charge * p.px[i] * psa_inv;
    T vy = p.charge * p.py[i] * psa_inv;
    T vz = p.charge * p.pz[i] * psa_inv;
    W9<T> w = weights(p.dx[i], p.dy[i]);
    T* js[3] = {jx, jy, jz};
    T vs[3] = {vx, vy, vz};
    for (int c = 0; c < 3; ++c) {
      T* j = js[c];
      T v = vs[c];
      j[ijm1 + ix - 1] += w.w00 * v;
      j[ijm1 + ix] += w.w01 * v;
      j[ijm1 + ix + 1] += w.w02 * v;
      j[ij + ix - 1] += w.w10 * v;
      j[ij + ix] += w.w11 * v;
      j[ij + ix + 1] += w.w12 * v;
      j[ijp1 + ix - 1] += w.w20 * v;
      j[ijp1 + ix] += w.w21 * v;
      j[ijp1 + ix + 1] += w.w22 * v;
    }
  }
  return OK;
}

// src/lib.rs:395-476 (serial, particle order)
template <typename T>
static int calc_density(const Prtl<T>& p, const Sim<T>& s, Flds<T>& f) {
  T* dsty = f.dsty.spatial.data();
  T* dens = f.dens.spatial.data();
  const size_t len = f.dsty.spatial.size(), W = 2 + s.size_x;
  const size_t n = p.ix.size();
  const T q = p.charge;
  for (size_t i = 0; i < n; ++i) {
    size_t ix = p.ix[i], iy = p.iy[i];
    if (iy == 0 || ix == 0) return E_BOUNDS;
    size_t ijm1 = (iy - 1) * W, ij = iy * W, ijp1 = (iy + 1) * W;
    if (!(ijp1 + ix + 1 < len)) return E_BOUNDS;
    W9<T> w = weights(p.dx[i], p.dy[i]);
    dsty[ijm1 + ix - 1] += w.w00 * q;
    dsty[ijm1 + ix] += w.w01 * q;
    dsty[ijm1 + ix + 1] += w.w02 * q;
    dsty[ij + ix - 1] += w.w10 * q;
    dsty[ij + ix] += w.w11 * q;
    dsty[ij + ix + 1] += w.w12 * q;
    dsty[ijp1 + ix - 1] += w.w20 * q;
    dsty[ijp1 + ix] += w.w21 * q;
    dsty[ijp1 + ix + 1] += w.w22 * q;
    dens[ijm1 + ix - 1] += w.w00;
    dens[ijm1 + ix] += w.w01;
    dens[ijm1 + ix + 1] += w.w02;
    dens[ij + ix - 1] += w.w10;
    dens[ij + ix] += w.w11;
    dens[ij + ix + 1] += w.w12;
    dens[ijp1 + ix - 1] += w.w20;
    dens[ijp1 + ix] += w.w21;
    dens[ijp1 + ix + 1] += w.w22;
  }
  return OK;
}

// src/lib.rs:478-489
template <typename T>
static int move_and_deposit(Prtl<T>& p, const Sim<T>& s, Flds<T>& f) {
  int e;
  if ((e = update_position(p, s))) return e;
  if ((e = apply_bc(p, s))) return e;
  if ((e = deposit_current(p, s, f))) return e;
  if ((e = update_position(p, s))) return e;
  if ((e = apply_bc(p, s))) return e;
  return calc_density(p, s, f);
}

// src/prtls.rs:262-443 (parallel in chunks of PRTL_CHUNK_SIZE)
template <typename T>
static int boris_push(Prtl<T>& p, const Sim<T>& s, const Flds<T>& f) {
  const T csqinv = T(1.) / (s.c * s.c);
  const T beta = p.beta, alpha = p.alpha;
  const T* E[3] = {f.e_x.spatial.data(), f.e_y.spatial.data(), f.e_z.spatial.data()};
  const T* B[3] = {f.b_x.spatial.data(), f.b_y.spatial.data(), f.b_z.spatial.data()};
  const size_t len = f.e_x.spatial.size(), W = 2 + s.size_x;
  const size_t n = p.ix.size();
  int err = OK;
  const long nchunks = (long)((n + PRTL_CHUNK_SIZE - 1) / PRTL_CHUNK_SIZE);
#pragma omp parallel for schedule(dynamic, 1) reduction(max : err)
  for (long ch = 0; ch < nchunks; ++ch) {
    size_t i0 = (size_t)ch * PRTL_CHUNK_SIZE, i1 = std::min(n, i0 + PRTL_CHUNK_SIZE);
    for (size_t i = i0; i < i1; ++i) {
      size_t ix = p.ix[i], iy = p.iy[i];
      if (iy == 0 || ix == 0 || !((iy + 1) * W + ix + 1 < len)) {
        err = E_BOUNDS;
        continue;
      }
      size_t ijm1 = (iy - 1) * W, ij = iy * W, ijp1 = (iy + 1) * W;
      W9<T> w = weights(p.dx[i], p.dy[i]);
      T g[6];
      for (int c = 0; c < 6; ++c) {
        const T* a = c < 3 ? E[c] : B[c - 3];
        T t = w.w00 * a[ijm1 + ix - 1];
        t += w.w01 * a[ijm1 + ix];
        t += w.w02 * a[ijm1 + ix + 1];
        t += w.w10 * a[ij + ix - 1];
        t += w.w11 * a[ij + ix];
        t += w.w12 * a[ij + ix + 1];
        t += w.w20 * a[ijp1 + ix - 1];
        t += w.w21 * a[ijp1 + ix];
        t += w.w22 * a[ijp1 + ix + 1];
        g[c] = t;
      }
      T ext = g[0] * beta, eyt = g[1] * beta, ezt = g[2] * beta;
      T bxt = g[3] * alpha, byt = g[4] * alpha, bzt = g[5] * alpha;
      T ux = p.px[i] + ext;
      T uy = p.py[i] + eyt;
      T uz = p.pz[i] + ezt;
      T gt = T(1) / std::sqrt(T(1.) + (ux * ux + uy * uy + uz * uz) * csqinv);
      bxt *= gt;
      byt *= gt;
      bzt *= gt;
      T boris = T(2.0) * (T(1) / (T(1.0) + bxt * bxt + byt * byt + bzt * bzt));
      T uxt = ux + uy * bzt - uz * byt;
      T uyt = uy + uz * bxt - ux * bzt;
      T uzt = uz + ux * byt - uy * bxt;
      p.px[i] = ux + boris * (uyt * bzt - uzt * byt) + ext;
      p.py[i] = uy + boris * (uzt * bxt - uxt * bzt) + eyt;
      p.pz[i] = uz + boris * (uxt * byt - uyt * bxt) + ezt;
      p.psa[i] = std::sqrt(T(1.0) + (p.px[i] * p.px[i] + p.py[i] * p.py[i] + p.pz[i] * p.pz[i]) * csqinv);
    }
  }
  return err;
}

// ---------------------------------------------------------------- context
template <typename T>
struct Ctx {
  Sim<T> sim;
  Flds<T> flds;
  std::vector<Prtl<T>> prtls;
  uint32_t t = 0;
};

}  // namespace orc

using namespace orc;

// ======================================================================
// C ABI for ctypes.  Every call returns 0 on success.  `_f32` entry points
// run the reference FP32 path, `_f64` the dprec path.  Host arrays are
// caller-owned and copied.
// ======================================================================
struct orc_params {
  uint64_t size_x, size_y, delta;
  double dt, c;
  uint32_t dens;
  double gamma_inj;
  uint32_t n_pass;
  int32_t periodic_x;
  int32_t left_wall;
};

#define ORC_API extern "C" __attribute__((visibility("default")))

template <typename T>
static Ctx<T>* make_ctx(const orc_params* p) {
  if (!p || p->size_x < 2 || p->size_y < 2 || p->dens == 0) return nullptr;
  auto* c = new Ctx<T>();
  c->sim.size_x = p->size_x;
  c->sim.size_y = p->size_y;
  c->sim.delta = p->delta;
  c->sim.dt = (T)p->dt;
  c->sim.c = (T)p->c;
  c->sim.dens = p->dens;
  c->sim.gamma_inj = (T)p->gamma_inj;
  c->sim.n_pass = p->n_pass;
  c->sim.periodic_x = p->periodic_x != 0;
  c->sim.left_wall = p->left_wall != 0;
  c->flds.init(c->sim);
  return c;
}

template <typename T>
static int add_species(Ctx<T>* c, double charge, double mass, double vth, uint64_t n, const uint64_t* ix,
                       const uint64_t* iy, const T* dx, const T* dy, const T* px, const T* py, const T* pz,
                       const T* psa) {
  if (!c) return E_ARG;
  Prtl<T> p;
  T q = (T)charge, m = (T)mass;
  // prtls.rs:61-62
  p.beta = (q / m) * T(0.5) * c->sim.dt;
  p.alpha = (q / m) * T(0.5) * c->sim.dt / c->sim.c;
  p.charge = q;
  p.vth = (T)vth;
  p.ix.assign(ix, ix + n);
  p.iy.assign(iy, iy + n);
  p.dx.assign(dx, dx + n);
  p.dy.assign(dy, dy + n);
  p.px.assign(px, px + n);
  p.py.assign(py, py + n);
  p.pz.assign(pz, pz + n);
  p.psa.assign(psa, psa + n);
  c->prtls.push_back(std::move(p));
  return OK;
}

template <typename T>
static int get_species(Ctx<T>* c, int s, uint64_t* ix, uint64_t* iy, T* dx, T* dy, T* px, T* py, T* pz,
                       T* psa) {
  if (!c || s < 0 || s >= (int)c->prtls.size()) return E_ARG;
  const Prtl<T>& p = c->prtls[s];
  size_t n = p.ix.size();
  std::copy(p.ix.begin(), p.ix.end(), ix);
  std::copy(p.iy.begin(), p.iy.end(), iy);
  std::memcpy(dx, p.dx.data(), n * sizeof(T));
  std::memcpy(dy, p.dy.data(), n * sizeof(T));
  std::memcpy(px, p.px.data(), n * sizeof(T));
  std::memcpy(py, p.py.data(), n * sizeof(T));
  std::memcpy(pz, p.pz.data(), n * sizeof(T));
  std::memcpy(psa, p.psa.data(), n * sizeof(T));
  return OK;
}

template <typename T>
static void zero_sources(Ctx<T>* c) {
  for (Field<T>* f : {&c->flds.j_x, &c->flds.j_y, &c->flds.j_z, &c->flds.dsty, &c->flds.dens})
    std::fill(f->spatial.begin(), f->spatial.end(), T(0));
}

template <typename T>
static void fold_sources(Ctx<T>* c) {
  for (Field<T>* f : {&c->flds.j_x, &c->flds.j_y, &c->flds.j_z, &c->flds.dsty, &c->flds.dens})
    deposit_ghosts(f->spatial, c->sim.size_x, c->sim.size_y);
}

// lib.rs:130-142: the extra move+deposit before the loop
template <typename T>
static int prepare(Ctx<T>* c) {
  for (auto& p : c->prtls) {
    int e = move_and_deposit(p, c->sim, c->flds);
    if (e) return e;
  }
  fold_sources(c);
  return OK;
}

// lib.rs:151-200, one iteration (without save_output)
template <typename T>
static int step(Ctx<T>* c) {
  zero_sources(c);
  for (auto& p : c->prtls) {
    int e = move_and_deposit(p, c->sim, c->flds);
    if (e) return e;
  }
  fold_sources(c);
  c->flds.update(c->sim);
  for (auto& p : c->prtls) {
    int e = boris_push(p, c->sim, c->flds);
    if (e) return e;
  }
  c->t += 1;
  return OK;
}

#define ORC_DEFINE(SUF, T)                                                                                 \
  ORC_API void* orc_create_##SUF(const orc_params* p) { return make_ctx<T>(p); }                           \
  ORC_API void orc_destroy_##SUF(void* c) { delete (Ctx<T>*)c; }                                           \
  ORC_API int orc_add_species_##SUF(void* c, double q, double m, double vth, uint64_t n, const uint64_t* ix, \
                                    const uint64_t* iy, const T* dx, const T* dy, const T* px, const T* py, \
                                    const T* pz, const T* psa) {                                           \
    return add_species<T>((Ctx<T>*)c, q, m, vth, n, ix, iy, dx, dy, px, py, pz, psa);                      \
  }                                                                                                        \
  ORC_API int orc_get_species_##SUF(void* c, int s, uint64_t* ix, uint64_t* iy, T* dx, T* dy, T* px, T* py, \
                                    T* pz, T* psa) {                                                       \
    return get_species<T>((Ctx<T>*)c, s, ix, iy, dx, dy, px, py, pz, psa);                                 \
  }                                                                                                        \
  ORC_API int orc_move_and_deposit_##SUF(void* cv, int s) {                                                \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    if (!c || s < 0 || s >= (int)c->prtls.size()) return E_ARG;                                            \
    return move_and_deposit(c->prtls[s], c->sim, c->flds);                                                 \
  }                                                                                                        \
  ORC_API int orc_boris_push_##SUF(void* cv, int s) {                                                      \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    if (!c || s < 0 || s >= (int)c->prtls.size()) return E_ARG;                                            \
    return boris_push(c->prtls[s], c->sim, c->flds);                                                       \
  }                                                                                                        \
  ORC_API int orc_zero_sources_##SUF(void* c) {                                                            \
    zero_sources<T>((Ctx<T>*)c);                                                                           \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_fold_sources_##SUF(void* c) {                                                            \
    fold_sources<T>((Ctx<T>*)c);                                                                           \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_fields_update_##SUF(void* cv) {                                                          \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    c->flds.update(c->sim);                                                                                \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_prepare_##SUF(void* c) { return prepare<T>((Ctx<T>*)c); }                                \
  ORC_API int orc_step_##SUF(void* cv, uint32_t n) {                                                       \
    for (uint32_t k = 0; k < n; ++k) {                                                                     \
      int e = step<T>((Ctx<T>*)cv);                                                                        \
      if (e) return e;                                                                                     \
    }                                                                                                      \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_get_field_##SUF(void* cv, int id, T* out) {                                              \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    Field<T>* f = c ? c->flds.by_id(id) : nullptr;                                                         \
    if (!f) return E_ARG;                                                                                  \
    std::memcpy(out, f->spatial.data(), f->spatial.size() * sizeof(T));                                    \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_set_field_##SUF(void* cv, int id, const T* in) {                                         \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    Field<T>* f = c ? c->flds.by_id(id) : nullptr;                                                         \
    if (!f) return E_ARG;                                                                                  \
    std::memcpy(f->spatial.data(), in, f->spatial.size() * sizeof(T));                                     \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_get_bwrk_##SUF(void* cv, int comp, T* out) {                                             \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    if (!c || comp < 0 || comp > 2) return E_ARG;                                                          \
    auto& w = comp == 0 ? c->flds.b_x_wrk : comp == 1 ? c->flds.b_y_wrk : c->flds.b_z_wrk;                 \
    std::memcpy(out, w.data(), w.size() * sizeof(Cx<T>));                                                  \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_set_bwrk_##SUF(void* cv, int comp, const T* in) {                                        \
    Ctx<T>* c = (Ctx<T>*)cv;                                                                               \
    if (!c || comp < 0 || comp > 2) return E_ARG;                                                          \
    auto& w = comp == 0 ? c->flds.b_x_wrk : comp == 1 ? c->flds.b_y_wrk : c->flds.b_z_wrk;                 \
    std::memcpy(w.data(), in, w.size() * sizeof(Cx<T>));                                                   \
    return 0;                                                                                              \
  }                                                                                                        \
  /* standalone field ops on caller arrays (golden-vector tests) */                                        \
  ORC_API int orc_field_op_##SUF(uint64_t nx, uint64_t ny, int op, T* spatial, uint32_t n_pass) {          \
    std::vector<T> f(spatial, spatial + (nx + 2) * (ny + 2));                                              \
    if (op == 0)                                                                                           \
      deposit_ghosts(f, nx, ny);                                                                           \
    else if (op == 1)                                                                                      \
      update_ghosts(f, nx, ny);                                                                            \
    else if (op == 2) {                                                                                    \
      std::vector<T> w(f.size(), T(0));                                                                    \
      for (uint32_t k = 0; k < n_pass; ++k) binomial_filter_2_d(f, w, nx, ny);                             \
    } else                                                                                                 \
      return E_ARG;                                                                                        \
    std::memcpy(spatial, f.data(), f.size() * sizeof(T));                                                  \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_copy_to_spectral_##SUF(uint64_t nx, uint64_t ny, const T* spatial, T* spectral) {        \
    Field<T> f;                                                                                            \
    f.init(nx, ny);                                                                                        \
    std::memcpy(f.spatial.data(), spatial, f.spatial.size() * sizeof(T));                                  \
    copy_to_spectral(f);                                                                                   \
    std::memcpy(spectral, f.spectral.data(), f.spectral.size() * sizeof(Cx<T>));                           \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_copy_to_spatial_##SUF(uint64_t nx, uint64_t ny, const T* spectral, T* spatial) {         \
    Field<T> f;                                                                                            \
    f.init(nx, ny);                                                                                        \
    std::memcpy(f.spectral.data(), spectral, f.spectral.size() * sizeof(Cx<T>));                           \
    copy_to_spatial(f);                                                                                    \
    std::memcpy(spatial, f.spatial.data(), f.spatial.size() * sizeof(T));                                  \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_fft2d_##SUF(uint64_t nx, uint64_t ny, T* data, int inverse) {                            \
    Plan1D px, py;                                                                                         \
    px.init(nx);                                                                                           \
    py.init(ny);                                                                                           \
    std::vector<Cx<T>> a((Cx<T>*)data, (Cx<T>*)data + nx * ny);                                            \
    fft2d(a, nx, ny, px, py, inverse != 0);                                                                \
    std::memcpy(data, a.data(), a.size() * sizeof(Cx<T>));                                                 \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_fft1d_##SUF(uint64_t n, T* data, int inverse) {                                          \
    Plan1D p;                                                                                              \
    p.init(n);                                                                                             \
    std::vector<double> re(n), im(n);                                                                      \
    for (size_t i = 0; i < n; ++i) {                                                                       \
      re[i] = data[2 * i];                                                                                 \
      im[i] = data[2 * i + 1];                                                                             \
    }                                                                                                      \
    p.run(re, im, inverse ? +1 : -1);                                                                      \
    for (size_t i = 0; i < n; ++i) {                                                                       \
      data[2 * i] = (T)re[i];                                                                              \
      data[2 * i + 1] = (T)im[i];                                                                          \
    }                                                                                                      \
    return 0;                                                                                              \
  }                                                                                                        \
  ORC_API int orc_wave_numbers_##SUF(uint64_t nx, uint64_t ny, T* kx, T* ky, T* kn) {                      \
    std::vector<T> a, b, c;                                                                                \
    wave_numbers<T>(nx, ny, a, b, c);                                                                      \
    std::memcpy(kx, a.data(), a.size() * sizeof(T));                                                       \
    std::memcpy(ky, b.data(), b.size() * sizeof(T));                                                       \
    std::memcpy(kn, c.data(), c.size() * sizeof(T));                                                       \
    return 0;                                                                                              \
  }

ORC_DEFINE(f32, float)
ORC_DEFINE(f64, double)

// Momentum initialisation of src/prtls.rs:222-250, fed with caller-supplied
// random draws (the reference uses an unseeded thread_rng; the build draws a
// seeded stream once and gives the same numbers to every path).
//   normals: 3 per particle (StandardNormal), uniforms: 1 per particle in [0,1).
//   beta_sign: +1 drifts along +x as in the reference, -1 along -x.
template <typename T>
static void init_velocities(uint64_t n, T c, T vth, T gamma_inj, T beta_sign, const T* normals,
                            const T* uniforms, T* px, T* py, T* pz, T* psa) {
  const T csqinv = T(1.) / (c * c);
  const T beta_inj = gamma_inj > T(1) ? beta_sign * std::sqrt(T(1.) - T(1) / (gamma_inj * gamma_inj)) : T(0);
  for (uint64_t i = 0; i < n; ++i) {
    px[i] = normals[3 * i + 0];
    px[i] *= vth * c;
    py[i] = normals[3 * i + 1];
    py[i] *= vth * c;
    pz[i] = normals[3 * i + 2];
    pz[i] *= vth * c;
    psa[i] = T(1.0) + (px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]) * csqinv;
    psa[i] = std::sqrt(psa[i]);
    if (!(gamma_inj > T(1))) continue;  // additive: no drift at all (the reference requires gamma_inj > 1)
    T ux = px[i] / c;
    T r = uniforms[i];
    if (-beta_inj * ux > r * psa[i]) ux *= T(-1.);
    px[i] = gamma_inj * (ux + beta_inj * psa[i]);
    px[i] *= c;
    psa[i] = T(1.0) + (px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]) * csqinv;
    psa[i] = std::sqrt(psa[i]);
  }
}

ORC_API int orc_init_velocities_f32(uint64_t n, double c, double vth, double g, double sgn, const float* nrm,
                                    const float* uni, float* px, float* py, float* pz, float* psa) {
  init_velocities<float>(n, (float)c, (float)vth, (float)g, (float)sgn, nrm, uni, px, py, pz, psa);
  return 0;
}
ORC_API int orc_init_velocities_f64(uint64_t n, double c, double vth, double g, double sgn, const double* nrm,
                                    const double* uni, double* px, double* py, double* pz, double* psa) {
  init_velocities<double>(n, c, vth, g, sgn, nrm, uni, px, py, pz, psa);
  return 0;
}

ORC_API int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
