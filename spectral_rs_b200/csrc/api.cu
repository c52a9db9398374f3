// C ABI of the B200 hot path (include/spectral_gpu.h): context, species
// management, the per-phase entry points and the graph-captured step.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "fields.cuh"
#include "particles.cuh"

using namespace spx;

struct StepGraph {
  cudaGraphExec_t exec;
  int launches;  // kernel launches it holds
};

// Upload of the caller's arrays: chunks of UPLOAD_CHUNK particles cross PCIe
// through two device buffers on a copy stream while the context's stream
// packs the previous chunk, so the copies run back to back at the link's rate.
// The buffers (and the packed cells of the species being added) are kept for
// later uploads and released with the context: allocating and releasing
// multi-GB staging per species cost more than the copies themselves, and a
// release alone took up to 1.6 s on a busy device.
constexpr uint64_t UPLOAD_CHUNK = 1ull << 22;  // particles per chunk
constexpr size_t UPLOAD_BYTES = 24;            // per particle and buffer: dx..pz + psa (>= ix + iy)
struct UploadRing {
  cudaStream_t cs = nullptr;
  cudaEvent_t ready[2] = {nullptr, nullptr}, done[2] = {nullptr, nullptr};
  unsigned char* buf[2] = {nullptr, nullptr};
  uint64_t chunk = 0;       // particles per buffer
  uint32_t* cell = nullptr;  // packed cells (ix | iy << 16) of the species being added
  uint64_t cell_n = 0;
  // room for a species of n particles in nbuf chunk buffers (cells: also the
  // packed-cell buffer of n)
  void reserve(uint64_t n, bool cells = true, int nbuf = 2) {
    if (!cs) {
      SPX_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      for (int b = 0; b < 2; ++b) {
        SPX_CUDA_TRY(cudaEventCreateWithFlags(&ready[b], cudaEventDisableTiming));
        SPX_CUDA_TRY(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming));
      }
    }
    const uint64_t m = std::max<uint64_t>(1, std::min(n, UPLOAD_CHUNK));
    if (m > chunk) {  // all buffers share one size
      SPX_CUDA_TRY(cudaStreamSynchronize(cs));
      for (int b = 0; b < 2; ++b) {
        if (buf[b]) SPX_CUDA_TRY(cudaFree(buf[b]));
        buf[b] = nullptr;
      }
      chunk = m;
    }
    for (int b = 0; b < nbuf; ++b)
      if (!buf[b]) SPX_CUDA_TRY(cudaMalloc(&buf[b], UPLOAD_BYTES * chunk));
    if (cells && std::max<uint64_t>(n, 1) > cell_n) {
      if (cell) SPX_CUDA_TRY(cudaFree(cell));
      cell = nullptr;
      cell_n = 0;
      SPX_CUDA_TRY(cudaMalloc(&cell, std::max<uint64_t>(n, 1) * 4));
      cell_n = std::max<uint64_t>(n, 1);
    }
  }
  void release() {
    if (cs) cudaStreamSynchronize(cs);
    for (int b = 0; b < 2; ++b) {
      if (buf[b]) cudaFree(buf[b]);
      if (ready[b]) cudaEventDestroy(ready[b]);
      if (done[b]) cudaEventDestroy(done[b]);
      buf[b] = nullptr;
      ready[b] = done[b] = nullptr;
    }
    if (cell) cudaFree(cell);
    if (cs) cudaStreamDestroy(cs);
    cs = nullptr;
    cell = nullptr;
    chunk = cell_n = 0;
  }
  // copy(off, m, buf, stream) queues the host-to-device copies of particles
  // [off, off + m); use(off, m, buf) queues the kernels that consume them on st.
  template <class Copy, class Use>
  void run(uint64_t n, cudaStream_t st, Copy copy, Use use) {
    // the first copies wait for everything already queued on st (a previous
    // pass may still read the buffers)
    SPX_CUDA_TRY(cudaEventRecord(done[0], st));
    SPX_CUDA_TRY(cudaStreamWaitEvent(cs, done[0], 0));
    uint64_t k = 0;
    for (uint64_t off = 0; off < n; off += chunk, ++k) {
      const int b = (int)(k & 1);
      const uint64_t m = std::min(chunk, n - off);
      if (k >= 2) SPX_CUDA_TRY(cudaStreamWaitEvent(cs, done[b], 0));
      copy(off, m, buf[b], cs);
      SPX_CUDA_TRY(cudaEventRecord(ready[b], cs));
      SPX_CUDA_TRY(cudaStreamWaitEvent(st, ready[b], 0));
      use(off, m, buf[b]);
      SPX_CUDA_TRY(cudaEventRecord(done[b], st));
    }
  }
};

struct spx_ctx {
  spx_params prm{};
  Grid g{};
  FieldBuffers fb;
  ParticleGeom pg;
  PhysParams pp{};
  std::vector<Species> species;
  cudaStream_t st = nullptr;
  int* d_err = nullptr;
  double* d_diag = nullptr;
  uint32_t* d_u32 = nullptr;  // scratch scalars
  uint32_t* d_counts = nullptr;
  bool pending_push = false;
  bool plain = false;
  std::string err;
  // graphs of one fused step, keyed by the species' buffer parities
  std::map<uint32_t, StepGraph> graphs;
  bool use_graphs = true;
  // timing ring
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // 5 per step
  int ev_steps = 0;
  float last_timing[4] = {0, 0, 0, 0};
  uint64_t last_launches = 0;
  uint64_t repacks = 0, last_overflow = 0, last_max_occ = 0;
  // Prtl::tag and Prtl::track (src/prtls.rs:21-22) per species.  Particles
  // never change their reference index, so these are fixed tables over it; an
  // empty table means the reference's defaults: tag[i] = i (src/prtls.rs:213),
  // only particle 40 tracked (src/prtls.rs:79).
  std::vector<std::vector<uint64_t>> tags;
  std::vector<std::vector<uint8_t>> track;
  std::vector<int32_t*> d_track_rank;  // output position of each tracked particle, -1 otherwise (lazy)
  std::vector<uint64_t> n_tracked;
  UploadRing own_up;         // spx_add_species scratch of a standalone context
  UploadRing* up = &own_up;  // the ring in use: a batch lends its one ring to every member
};

static std::string g_create_err;

static int fail(spx_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  else g_create_err = m;
  return code;
}

// Every call on a context runs on the context's device (the CUDA runtime's current
// device is per host thread).
#define SPX_GUARD(ctx, ...)                           \
  try {                                               \
    SPX_CUDA_TRY(cudaSetDevice((ctx)->prm.device));   \
    __VA_ARGS__;                                      \
  } catch (const spx::Error& e) {                     \
    return fail(ctx, e.code, e.msg);                  \
  } catch (const std::exception& e) {                 \
    return fail(ctx, SPX_ERR_CUDA, e.what());         \
  }

static int check_device_error(spx_ctx* c) {
  int h = 0;
  SPX_CUDA_TRY(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  if (!h) return SPX_OK;
  SPX_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
  if (h & DERR_WALL) return fail(c, SPX_ERR_WALL, "reflecting wall assertion: a particle is beyond wall_loc+1 or at ix <= delta");
  if (h & DERR_BOUNDS) return fail(c, SPX_ERR_BOUNDS, "particle cell index out of the grid");
  if (h & DERR_OVERFLOW_LOST) return fail(c, SPX_ERR_STATE, "particle overflow list full: slot capacity too small");
  if (h & DERR_TIMEOUT) return fail(c, SPX_ERR_TIMEOUT, "a bounded wait for staged particle data gave up");
  return fail(c, SPX_ERR_STATE, "device error word " + std::to_string(h));
}

static void invalidate_graphs(spx_ctx* c) {
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
  c->graphs.clear();
}

static FieldPtrs field_ptrs(spx_ctx* c) {
  FieldPtrs f;
  for (int i = 0; i < 3; ++i) {
    f.E[i] = c->fb.spatial[SPX_EX + i];
    f.B[i] = c->fb.spatial[SPX_BX + i];
    f.J[i] = c->fb.spatial[SPX_JX + i];
  }
  f.dsty = c->fb.spatial[SPX_DSTY];
  f.dens = c->fb.spatial[SPX_DENS];
  return f;
}

// ---------------------------------------------------------------- create / destroy
extern "C" int spx_create(const spx_params* p, spx_ctx** out) {
  if (!p || !out) return fail(nullptr, SPX_ERR_ARG, "null argument");
  *out = nullptr;
  if (p->size_x % 2 || p->size_y % 2) return fail(nullptr, SPX_ERR_ARG, "Number of cells must be even (src/lib.rs:76)");
  if (!is_pow2(p->size_x) || !is_pow2(p->size_y) || p->size_x < 8 || p->size_y < 8 || p->size_x > 8192 ||
      p->size_y > 8192)
    return fail(nullptr, SPX_ERR_ARG, "GPU FFT needs power-of-two sizes in [8, 8192]");
  if (!p->periodic_x && p->delta * 2 >= p->size_x)
    return fail(nullptr, SPX_ERR_ARG, "Delta must be less than 1/2 the size of size_x (src/lib.rs:88)");
  if (p->dens == 0 || !(p->c > 0) || !(p->dt > 0)) return fail(nullptr, SPX_ERR_ARG, "dens, c and dt must be positive");
  if (p->slot_headroom < 0 || p->slot_headroom > 64 || p->arrival_slots < 0 || p->arrival_slots > 4096)
    return fail(nullptr, SPX_ERR_ARG, "slot_headroom must be in [0, 64] and arrival_slots in [0, 4096]");
  spx_ctx* c = new spx_ctx();
  c->prm = *p;
  try {
    SPX_CUDA_TRY(cudaSetDevice(p->device));
    SPX_CUDA_TRY(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    c->g.nx = (int)p->size_x;
    c->g.ny = (int)p->size_y;
    c->g.W = c->g.nx + 2;
    c->g.log2nx = ilog2(p->size_x);
    c->g.log2ny = ilog2(p->size_y);
    c->fb.dt = p->dt;
    c->fb.c = p->c;
    c->fb.dens = p->dens;
    c->fb.n_pass = p->n_pass;
    c->fb.allocate(c->g);
    // tiles: power-of-two; 16 x 8 unless params set one (128-thread CTAs compiled for five
    // resident per SM, 20 warps: measured 1 % faster than 8 x 8 and 4-10 % faster than 16 x 16
    // on the thermal and Weibel plasmas; batches keep 8 x 8)
    int tx = p->tile_x > 0 ? p->tile_x : 16, ty = p->tile_y > 0 ? p->tile_y : 8;
    tx = std::min(tx, c->g.nx);
    ty = std::min(ty, c->g.ny);
    if (!is_pow2(tx) || !is_pow2(ty) || tx * ty > 256 || tx * ty < 32) {
      spx_destroy(c);  // releases the stream and fields allocated above
      return fail(nullptr, SPX_ERR_ARG, "tile_x*tile_y must be a power-of-two product in [32, 256]");
    }
    c->pg.g = c->g;
    c->pg.TX = tx;
    c->pg.TY = ty;
    c->pg.logTX = ilog2(tx);
    c->pg.logTY = ilog2(ty);
    c->pg.NTX = c->g.nx / tx;
    c->pg.NTY = c->g.ny / ty;
    c->pp.dt = p->dt;
    c->pp.c = p->c;
    c->pp.csqinv = 1.0f / (p->c * p->c);  // src/prtls.rs:265
    c->pp.periodic_x = p->periodic_x;
    c->pp.left_wall = p->left_wall;
    c->pp.wall_loc = (int)(p->size_x + 1 - p->delta);  // src/prtls.rs:153
    c->pp.delta = (int)p->delta;
    c->pp.compensated = p->compensated != 0;
    c->plain = p->path == SPX_PATH_PLAIN;
    SPX_CUDA_TRY(cudaMalloc(&c->d_err, sizeof(int)));
    SPX_CUDA_TRY(cudaMemset(c->d_err, 0, sizeof(int)));
    SPX_CUDA_TRY(cudaMalloc(&c->d_diag, 8 * sizeof(double)));
    SPX_CUDA_TRY(cudaMalloc(&c->d_u32, 8 * sizeof(uint32_t)));
    SPX_CUDA_TRY(cudaMalloc(&c->d_counts, c->pg.ncells() * sizeof(uint32_t)));
    slot_set_kernel_attributes();
    fields_set_kernel_attributes();
    // the zero fills above ran on the legacy stream, which the context's
    // non-blocking stream does not wait for
    SPX_CUDA_TRY(cudaDeviceSynchronize());
  } catch (const spx::Error& e) {
    spx_destroy(c);
    return fail(nullptr, e.code, e.msg);
  }
  *out = c;
  return SPX_OK;
}

extern "C" int spx_destroy(spx_ctx* c) {
  if (!c) return SPX_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  invalidate_graphs(c);
  for (auto& s : c->species) {
    slot_release(s);
    for (float* p : {s.plain.x, s.plain.y, s.plain.px, s.plain.py, s.plain.pz})
      if (p) cudaFree(p);
  }
  for (int32_t* p : c->d_track_rank)
    if (p) cudaFree(p);
  c->fb.release();
  c->own_up.release();
  for (void* p : {(void*)c->d_err, (void*)c->d_diag, (void*)c->d_u32, (void*)c->d_counts})
    if (p) cudaFree(p);
  for (auto e : c->ev) cudaEventDestroy(e);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return SPX_OK;
}

extern "C" const char* spx_last_error(const spx_ctx* c) { return c ? c->err.c_str() : g_create_err.c_str(); }

extern "C" const char* spx_version(void) {
  return "spectral_rs_b200 hot path: sm_100a, FP32, particle TU -fmad=false, IEEE div/sqrt";
}

extern "C" int32_t spx_num_species(const spx_ctx* c) { return c ? (int32_t)c->species.size() : 0; }
extern "C" uint64_t spx_species_count(const spx_ctx* c, int32_t s) {
  if (!c || s < 0 || s >= (int)c->species.size()) return 0;
  return c->species[s].n;
}

// ---------------------------------------------------------------- species upload
// Device staging of one species in the reference order, then packing.
struct Staging {
  uint32_t* cell = nullptr;
  float *dx = nullptr, *dy = nullptr, *px = nullptr, *py = nullptr, *pz = nullptr;
  void alloc(uint64_t n) {
    SPX_CUDA_TRY(cudaMalloc(&cell, std::max<uint64_t>(n, 1) * 4));
    SPX_CUDA_TRY(cudaMalloc(&dx, std::max<uint64_t>(n, 1) * 4));
    SPX_CUDA_TRY(cudaMalloc(&dy, std::max<uint64_t>(n, 1) * 4));
    SPX_CUDA_TRY(cudaMalloc(&px, std::max<uint64_t>(n, 1) * 4));
    SPX_CUDA_TRY(cudaMalloc(&py, std::max<uint64_t>(n, 1) * 4));
    SPX_CUDA_TRY(cudaMalloc(&pz, std::max<uint64_t>(n, 1) * 4));
  }
  ~Staging() {
    for (void* p : {(void*)cell, (void*)dx, (void*)dy, (void*)px, (void*)py, (void*)pz})
      if (p) cudaFree(p);
  }
};

__global__ void k_plain_from_cells(uint64_t n, const uint32_t* cell, const float* dx, const float* dy, float* x,
                                   float* y) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    x[i] = (float)(cell[i] & 0xFFFFu) + dx[i];
    y[i] = (float)(cell[i] >> 16) + dy[i];
  }
}

// Slot capacity per cell: the low range KL and the arrival regions H.
struct Capacity {
  int KL, H;
};

// Capacity for n particles whose fullest cell holds mx.
static Capacity capacity_for(const spx_ctx* c, uint64_t n, uint32_t mx) {
  // exact low range and one arrival slot (tests: every step overflows)
  if (c->prm.slot_capacity < 0) return {std::max((int)mx, -c->prm.slot_capacity), 1};
  const double mean = (double)n / (double)c->pg.ncells();
  // room for Poisson-like fluctuations of the occupancy; the overflow list and
  // repack handle anything beyond
  const double f = c->prm.slot_headroom > 0 ? (double)c->prm.slot_headroom : 1.25;
  int KL = (int)std::ceil(std::max(f * mx, mean + 8.0 * std::sqrt(mean))) + 8;
  // a reflecting wall piles incoming and reflected particles up (a shock
  // compresses the plasma about fourfold): by default leave room for that from the
  // start, four times the fullest cell (which already holds the Poisson excess)
  if (!c->prm.periodic_x && !(c->prm.slot_headroom > 0)) KL = std::max(KL, (int)std::ceil(4.0 * mx) + 8);
  if (c->prm.slot_capacity > 0) KL = std::max(KL, c->prm.slot_capacity);
  // arrivals of one step: a few per cent of the occupancy in a thermal plasma,
  // a few tens in a fast flow
  const int H = c->prm.arrival_slots > 0 ? c->prm.arrival_slots : std::max(16, (KL + 3) / 4);
  return {KL, H};
}

// Largest per-cell count of c->d_counts.
static uint32_t max_count(spx_ctx* c) {
  uint32_t mx = 0;
  SPX_CUDA_TRY(cudaMemsetAsync(c->d_u32, 0, sizeof(uint32_t), c->st));
  Species tmp;
  tmp.slot.nlow = c->d_counts;
  slot_max_occupancy(tmp, c->pg, c->d_u32, c->st);
  SPX_CUDA_TRY(cudaMemcpyAsync(&mx, c->d_u32, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
  SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  return mx;
}

static Capacity choose_capacity(spx_ctx* c, uint64_t n) { return capacity_for(c, n, max_count(c)); }


__global__ void k_check_cells(uint64_t n, const uint32_t* cell, int nx, int ny, int* derr) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(cell[i] & 0xFFFFu), iy = (int)(cell[i] >> 16);
    if (ix < 1 || ix > nx || iy < 1 || iy > ny) atomicOr(derr, DERR_BOUNDS);
  }
}

__global__ void k_check_gamma(uint64_t n, const float* px, const float* py, const float* pz, const float* psa,
                              float csqinv, int* derr) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float g = __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(px[i], px[i]),
                                                                             __fmul_rn(py[i], py[i])),
                                                                   __fmul_rn(pz[i], pz[i])),
                                                         csqinv)));
    if (g != psa[i]) atomicOr(derr, DERR_GAMMA);
  }
}

// Cell indices (1-based, usize in the reference) -> packed cell; the smallest
// index (off + i) of a particle outside the grid goes to *bad (initialised to ~0).
__global__ void k_pack_check(uint64_t n, uint64_t off, const uint64_t* ix, const uint64_t* iy, int nx, int ny,
                             uint32_t* cell, uint32_t* bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = ix[i], y = iy[i];
    if (x < 1 || y < 1 || x > (uint64_t)nx || y > (uint64_t)ny) {
      atomicMin(bad, (uint32_t)(off + i));
      cell[i] = 1u | (1u << 16);
    } else {
      cell[i] = (uint32_t)x | ((uint32_t)y << 16);
    }
  }
}

static void add_species_tables(spx_ctx* c, const Species& s) {
  c->species.push_back(s);
  c->tags.emplace_back();
  c->track.emplace_back();
  c->d_track_rank.push_back(nullptr);
  c->n_tracked.push_back(0);
}

extern "C" int spx_add_species(spx_ctx* c, float charge, float mass, float vth, uint64_t n, const uint64_t* ix,
                               const uint64_t* iy, const float* dx, const float* dy, const float* px, const float* py,
                               const float* pz, const float* psa, int32_t* species_out) {
  if (!c) return fail(nullptr, SPX_ERR_ARG, "null context");
  if ((int)c->species.size() >= MAX_SPECIES) return fail(c, SPX_ERR_ARG, "at most 4 species");
  if (n && (!ix || !iy || !dx || !dy || !px || !py || !pz)) return fail(c, SPX_ERR_ARG, "null particle array");
  if (n >= (1ull << 32)) return fail(c, SPX_ERR_ARG, "at most 2^32-1 particles per species");
  if (!(mass != 0.0f)) return fail(c, SPX_ERR_ARG, "mass must be non-zero");
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    Species s;
    s.charge = charge;
    s.mass = mass;
    s.vth = vth;
    // src/prtls.rs:61-62, FP32 left to right
    s.beta = (charge / mass) * 0.5f * c->prm.dt;
    s.alpha = (charge / mass) * 0.5f * c->prm.dt / c->prm.c;
    s.n = n;
    UploadRing& up = *c->up;
    up.reserve(n);
    uint32_t* const cell = up.cell;
    // pass 1: cell indices checked and packed on the device, occupancy per cell
    SPX_CUDA_TRY(cudaMemsetAsync(c->d_u32, 0xFF, sizeof(uint32_t), c->st));
    if (!c->plain) SPX_CUDA_TRY(cudaMemsetAsync(c->d_counts, 0, c->pg.ncells() * sizeof(uint32_t), c->st));
    up.run(
        n, c->st,
        [&](uint64_t off, uint64_t m, unsigned char* b, cudaStream_t cs) {
          SPX_CUDA_TRY(cudaMemcpyAsync(b, ix + off, m * 8, cudaMemcpyHostToDevice, cs));
          SPX_CUDA_TRY(cudaMemcpyAsync(b + m * 8, iy + off, m * 8, cudaMemcpyHostToDevice, cs));
        },
        [&](uint64_t off, uint64_t m, unsigned char* b) {
          const uint64_t* bx = reinterpret_cast<const uint64_t*>(b);
          k_pack_check<<<148 * 4, 256, 0, c->st>>>(m, off, bx, bx + m, c->g.nx, c->g.ny, cell + off, c->d_u32);
          if (!c->plain) slot_count(c->pg, m, cell + off, c->d_counts, c->st, false);
        });
    // the first bad index and (slots) the fullest cell's count, read back together below
    uint32_t hb[2] = {0, 0};
    if (!c->plain) {
      SPX_CUDA_TRY(cudaMemsetAsync(c->d_u32 + 1, 0, sizeof(uint32_t), c->st));
      Species tmp;
      tmp.slot.nlow = c->d_counts;
      slot_max_occupancy(tmp, c->pg, c->d_u32 + 1, c->st);
    }
    // the destination arrays are allocated while pass 1's copies run: the plain
    // arrays, or the slots for a bound on the occupancy of a uniform species,
    // replaced below only if the counts ask for more
    auto release = [&]() {
      slot_release(s);
      for (float** p : {&s.plain.x, &s.plain.y, &s.plain.px, &s.plain.py, &s.plain.pz}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
      }
    };
    Capacity guess{0, 0};
    if (c->plain) {
      for (float** p : {&s.plain.x, &s.plain.y, &s.plain.px, &s.plain.py, &s.plain.pz})
        SPX_CUDA_TRY(cudaMalloc(p, std::max<uint64_t>(n, 1) * 4));
    } else if (c->prm.slot_capacity >= 0) {
      // the largest occupancy of a uniform plasma of mean m over N cells stays below
      // m + sqrt(2 m ln N) (Poisson tail): slots for that are allocated while the copies
      // run (allocating GBs of slots costs about as long as copying the particles) and
      // replaced below only when the counts need more
      const double m = (double)n / (double)c->pg.ncells();
      const double ln = std::log(std::max(2.0, (double)c->pg.ncells()));
      guess = capacity_for(c, n, (uint32_t)std::ceil(m + std::sqrt(2.0 * m * ln) + 2.0));
      slot_allocate(s, c->pg, guess.KL, guess.H, n);
    }
    // (a read-back into pageable memory returns once the copy is done, so it comes after
    // the allocation)
    SPX_CUDA_TRY(cudaMemcpyAsync(hb, c->d_u32, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    const uint32_t bad = hb[0];
    if (bad != 0xFFFFFFFFu) {
      release();
      return fail(c, SPX_ERR_BOUNDS, "particle " + std::to_string(bad) + " outside the grid");
    }
    // pass 2: offsets and momenta into their slots (or the plain arrays)
    if (!c->plain) {
      const Capacity cap = capacity_for(c, n, hb[1]);
      if (cap.KL > guess.KL || cap.H > guess.H) {
        slot_release(s);
        slot_allocate(s, c->pg, std::max(cap.KL, guess.KL), std::max(cap.H, guess.H), n);
      }
      slot_scatter_begin(s, c->pg, c->d_counts, c->st);
    }
    up.run(
        n, c->st,
        [&](uint64_t off, uint64_t m, unsigned char* b, cudaStream_t cs) {
          const float* src[6] = {dx, dy, px, py, pz, psa};
          for (int f = 0; f < (psa ? 6 : 5); ++f)
            SPX_CUDA_TRY(cudaMemcpyAsync(b + f * m * 4, src[f] + off, m * 4, cudaMemcpyHostToDevice, cs));
        },
        [&](uint64_t off, uint64_t m, unsigned char* b) {
          const float* f = reinterpret_cast<const float*>(b);
          if (psa) k_check_gamma<<<148 * 4, 256, 0, c->st>>>(m, f + 2 * m, f + 3 * m, f + 4 * m, f + 5 * m,
                                                             c->pp.csqinv, c->d_err);
          if (c->plain) {
            k_plain_from_cells<<<148 * 4, 256, 0, c->st>>>(m, cell + off, f, f + m, s.plain.x + off, s.plain.y + off);
            float* const mom[3] = {s.plain.px, s.plain.py, s.plain.pz};
            for (int k = 0; k < 3; ++k)
              SPX_CUDA_TRY(cudaMemcpyAsync(mom[k] + off, f + (2 + k) * m, m * 4, cudaMemcpyDeviceToDevice, c->st));
          } else {
            slot_scatter_chunk(s, c->pg, m, (uint32_t)off, cell + off, f, f + m, f + 2 * m, f + 3 * m, f + 4 * m,
                               nullptr, c->d_counts, c->st);
          }
        });
    if (!c->plain) slot_scatter_end(s, c->pg, c->d_counts, c->st);
    SPX_CUDA_TRY(cudaGetLastError());
    int h = 0;
    SPX_CUDA_TRY(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    if (h & DERR_GAMMA) {
      SPX_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st));
      release();
      return fail(c, SPX_ERR_GAMMA, "psa differs from sqrt(1 + |p|^2/c^2); the GPU derives gamma from p");
    }
    add_species_tables(c, s);
    if (species_out) *species_out = (int32_t)c->species.size() - 1;
    invalidate_graphs(c);
  });
  return SPX_OK;
}

extern "C" int spx_init_species(spx_ctx* c, float charge, float mass, float vth, uint32_t ppc, uint64_t x0,
                                uint64_t x1, float gamma_drift, float sign_x, int32_t random_positions,
                                uint64_t seed, int32_t* species_out) {
  if (!c) return fail(nullptr, SPX_ERR_ARG, "null context");
  if ((int)c->species.size() >= MAX_SPECIES) return fail(c, SPX_ERR_ARG, "at most 4 species");
  if (x1 > (uint64_t)c->g.nx || x0 >= x1 || ppc == 0) return fail(c, SPX_ERR_ARG, "bad column range or ppc");
  if (!(mass != 0.0f)) return fail(c, SPX_ERR_ARG, "mass must be non-zero");
  const uint64_t n = (uint64_t)c->g.ny * (x1 - x0) * ppc;
  if (n >= (1ull << 32)) return fail(c, SPX_ERR_ARG, "at most 2^32-1 particles per species");
  SPX_GUARD(c, {
    if (spx_flush(c) != SPX_OK) return SPX_ERR_STATE;
    Species s;
    s.charge = charge;
    s.mass = mass;
    s.vth = vth;
    s.beta = (charge / mass) * 0.5f * c->prm.dt;
    s.alpha = (charge / mass) * 0.5f * c->prm.dt / c->prm.c;
    s.n = n;
    InitSpec is;
    is.charge = charge;
    is.mass = mass;
    is.vth = vth;
    is.gamma_drift = gamma_drift;
    is.sign_x = sign_x;
    is.c = c->prm.c;
    is.ppc = ppc;
    is.x0 = (int)x0;
    is.x1 = (int)x1;
    is.random_positions = random_positions;
    is.seed = seed;
    // generated chunk by chunk into the upload ring and placed at once: every
    // cell of columns [x0, x1) holds exactly ppc particles, so the slot capacity
    // is known before the first particle exists
    UploadRing& up = *c->up;
    up.reserve(n, false, 1);
    if (c->plain) {
      for (float** p : {&s.plain.x, &s.plain.y, &s.plain.px, &s.plain.py, &s.plain.pz})
        SPX_CUDA_TRY(cudaMalloc(p, std::max<uint64_t>(n, 1) * 4));
    } else {
      const Capacity cap = capacity_for(c, n, ppc);
      slot_allocate(s, c->pg, cap.KL, cap.H, n);
      slot_scatter_begin(s, c->pg, c->d_counts, c->st);
    }
    for (uint64_t off = 0; off < n; off += up.chunk) {  // one stream, one buffer: chunks in order
      const uint64_t m = std::min(up.chunk, n - off);
      uint32_t* cl = reinterpret_cast<uint32_t*>(up.buf[0]);
      float* f = reinterpret_cast<float*>(up.buf[0]) + m;  // dx, dy, px, py, pz after the cells
      init_particles(is, c->g, off, m, cl, f, f + m, f + 2 * m, f + 3 * m, f + 4 * m, c->st);
      if (c->plain) {
        k_plain_from_cells<<<148 * 4, 256, 0, c->st>>>(m, cl, f, f + m, s.plain.x + off, s.plain.y + off);
        float* const mom[3] = {s.plain.px, s.plain.py, s.plain.pz};
        for (int k = 0; k < 3; ++k)
          SPX_CUDA_TRY(cudaMemcpyAsync(mom[k] + off, f + (2 + k) * m, m * 4, cudaMemcpyDeviceToDevice, c->st));
      } else {
        slot_scatter_chunk(s, c->pg, m, (uint32_t)off, cl, f, f + m, f + 2 * m, f + 3 * m, f + 4 * m, nullptr,
                           c->d_counts, c->st);
      }
    }
    if (!c->plain) slot_scatter_end(s, c->pg, c->d_counts, c->st);
    SPX_CUDA_TRY(cudaGetLastError());
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    add_species_tables(c, s);
    if (species_out) *species_out = (int32_t)c->species.size() - 1;
    invalidate_graphs(c);
  });
  return SPX_OK;
}

// ---------------------------------------------------------------- species download
__global__ void k_stride_u32(const uint32_t* in, uint64_t n, uint64_t stride, uint64_t* out) {
  const uint64_t m = (n + stride - 1) / stride;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i * stride];
}
__global__ void k_stride_f32(const float* in, uint64_t n, uint64_t stride, float* out) {
  const uint64_t m = (n + stride - 1) / stride;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i * stride];
}
__global__ void k_plain_to_cells(uint64_t n, const float* x, const float* y, uint32_t* ix, uint32_t* iy, float* dx,
                                 float* dy) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int cx = (int)floorf(x[i] + 0.5f), cy = (int)floorf(y[i] + 0.5f);
    ix[i] = (uint32_t)cx;
    iy[i] = (uint32_t)cy;
    dx[i] = x[i] - (float)cx;
    dy[i] = y[i] - (float)cy;
  }
}
// psa = sqrt(1 + |p|^2 / c^2) in the reference's rounding (src/prtls.rs:440): no contraction
__global__ void k_gamma_arr(uint64_t n, const float* px, const float* py, const float* pz, float csqinv, float* g) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    g[i] = __fsqrt_rn(__fadd_rn(1.0f, __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(px[i], px[i]), __fmul_rn(py[i], py[i])),
                                                          __fmul_rn(pz[i], pz[i])),
                                                csqinv)));
}

extern "C" int spx_get_species(spx_ctx* c, int32_t sidx, uint64_t stride, uint64_t* ix, uint64_t* iy, float* dx,
                               float* dy, float* px, float* py, float* pz, float* psa) {
  if (!c) return fail(nullptr, SPX_ERR_ARG, "null context");
  if (sidx < 0 || sidx >= (int)c->species.size()) return fail(c, SPX_ERR_ARG, "no such species");
  if (stride == 0) stride = 1;
  SPX_GUARD(c, {
    int e = spx_flush(c);
    if (e) return e;
    Species& s = c->species[sidx];
    const uint64_t n = s.n;
    const uint64_t m = (n + stride - 1) / stride;
    if (n == 0) return SPX_OK;
    uint32_t *d_ix, *d_iy;
    float *d_dx, *d_dy, *d_px, *d_py, *d_pz, *d_g;
    SPX_CUDA_TRY(cudaMallocAsync(&d_ix, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_iy, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_dx, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_dy, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_px, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_py, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_pz, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_g, n * 4, c->st));
    if (c->plain) {
      k_plain_to_cells<<<148 * 8, 256, 0, c->st>>>(n, s.plain.x, s.plain.y, d_ix, d_iy, d_dx, d_dy);
      SPX_CUDA_TRY(cudaMemcpyAsync(d_px, s.plain.px, n * 4, cudaMemcpyDeviceToDevice, c->st));
      SPX_CUDA_TRY(cudaMemcpyAsync(d_py, s.plain.py, n * 4, cudaMemcpyDeviceToDevice, c->st));
      SPX_CUDA_TRY(cudaMemcpyAsync(d_pz, s.plain.pz, n * 4, cudaMemcpyDeviceToDevice, c->st));
      k_gamma_arr<<<148 * 8, 256, 0, c->st>>>(n, d_px, d_py, d_pz, c->pp.csqinv, d_g);
    } else {
      slot_unpack(s, c->pg, d_ix, d_iy, d_dx, d_dy, d_px, d_py, d_pz, d_g, c->pp.csqinv, c->st);
    }
    // stride on the device, then copy out
    uint64_t* d_u64;
    float* d_f;
    SPX_CUDA_TRY(cudaMallocAsync(&d_u64, m * 8, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_f, m * 4, c->st));
    const int blocks = 148 * 8;
    if (ix) {
      k_stride_u32<<<blocks, 256, 0, c->st>>>(d_ix, n, stride, d_u64);
      SPX_CUDA_TRY(cudaMemcpyAsync(ix, d_u64, m * 8, cudaMemcpyDeviceToHost, c->st));
      SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    if (iy) {
      k_stride_u32<<<blocks, 256, 0, c->st>>>(d_iy, n, stride, d_u64);
      SPX_CUDA_TRY(cudaMemcpyAsync(iy, d_u64, m * 8, cudaMemcpyDeviceToHost, c->st));
      SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    const float* srcs[6] = {d_dx, d_dy, d_px, d_py, d_pz, d_g};
    float* dsts[6] = {dx, dy, px, py, pz, psa};
    for (int k = 0; k < 6; ++k) {
      if (!dsts[k]) continue;
      k_stride_f32<<<blocks, 256, 0, c->st>>>(srcs[k], n, stride, d_f);
      SPX_CUDA_TRY(cudaMemcpyAsync(dsts[k], d_f, m * 4, cudaMemcpyDeviceToHost, c->st));
      SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    }
    for (void* p : {(void*)d_ix, (void*)d_iy, (void*)d_dx, (void*)d_dy, (void*)d_px, (void*)d_py, (void*)d_pz,
                    (void*)d_g, (void*)d_u64, (void*)d_f})
      SPX_CUDA_TRY(cudaFreeAsync(p, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

// ---------------------------------------------------------------- tags and tracked particles
extern "C" int spx_set_tags(spx_ctx* c, int32_t sidx, const uint64_t* tag, const uint8_t* track) {
  if (!c) return fail(nullptr, SPX_ERR_ARG, "null context");
  if (sidx < 0 || sidx >= (int)c->species.size()) return fail(c, SPX_ERR_ARG, "no such species");
  const uint64_t n = c->species[sidx].n;
  if (tag) c->tags[sidx].assign(tag, tag + n);
  if (track) {
    c->track[sidx].assign(track, track + n);
    if (c->d_track_rank[sidx]) cudaFree(c->d_track_rank[sidx]);
    c->d_track_rank[sidx] = nullptr;  // rebuilt by the next spx_get_tracked
  }
  return SPX_OK;
}

extern "C" int spx_get_tags(spx_ctx* c, int32_t sidx, uint64_t stride, uint64_t* tag, uint8_t* track) {
  if (!c) return fail(nullptr, SPX_ERR_ARG, "null context");
  if (sidx < 0 || sidx >= (int)c->species.size()) return fail(c, SPX_ERR_ARG, "no such species");
  if (stride == 0) stride = 1;
  const uint64_t n = c->species[sidx].n;
  const std::vector<uint64_t>& tg = c->tags[sidx];
  const std::vector<uint8_t>& tr = c->track[sidx];
  for (uint64_t i = 0, k = 0; i < n; i += stride, ++k) {
    if (tag) tag[k] = tg.empty() ? i : tg[i];
    if (track) track[k] = tr.empty() ? (uint8_t)(i == 40) : tr[i];
  }
  return SPX_OK;
}

extern "C" int spx_get_tracked(spx_ctx* c, int32_t sidx, uint64_t capacity, float* x, float* y, float* gamma,
                               uint64_t* count) {
  if (!c || !count) return fail(c, SPX_ERR_ARG, "null argument");
  if (sidx < 0 || sidx >= (int)c->species.size()) return fail(c, SPX_ERR_ARG, "no such species");
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    const Species& s = c->species[sidx];
    if (!c->d_track_rank[sidx]) {  // output position of every tracked particle, reference order
      std::vector<int32_t> rank(std::max<uint64_t>(s.n, 1), -1);
      const std::vector<uint8_t>& tr = c->track[sidx];
      uint64_t k = 0;
      for (uint64_t i = 0; i < s.n; ++i)
        if (tr.empty() ? i == 40 : tr[i] != 0) rank[i] = (int32_t)k++;
      SPX_CUDA_TRY(cudaMalloc(&c->d_track_rank[sidx], rank.size() * sizeof(int32_t)));
      SPX_CUDA_TRY(cudaMemcpy(c->d_track_rank[sidx], rank.data(), rank.size() * sizeof(int32_t),
                              cudaMemcpyHostToDevice));
      c->n_tracked[sidx] = k;
    }
    const uint64_t k = c->n_tracked[sidx];
    *count = k;
    if (k == 0 || (!x && !y && !gamma)) return SPX_OK;  // nothing tracked, or a count query
    if (k > capacity) return fail(c, SPX_ERR_ARG, "output capacity below the number of tracked particles");
    float* d_out;
    SPX_CUDA_TRY(cudaMallocAsync(&d_out, 3 * k * sizeof(float), c->st));
    gather_tracked(s, c->pg, c->plain, c->d_track_rank[sidx], c->prm.c, d_out, d_out + k, d_out + 2 * k, c->st);
    float* const dst[3] = {x, y, gamma};
    for (int f = 0; f < 3; ++f)
      if (dst[f]) SPX_CUDA_TRY(cudaMemcpyAsync(dst[f], d_out + f * k, k * sizeof(float), cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaFreeAsync(d_out, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

// ---------------------------------------------------------------- per-phase calls
static void zero_sources(spx_ctx* c) {
  for (int f : {SPX_JX, SPX_JY, SPX_JZ, SPX_DSTY, SPX_DENS})
    SPX_CUDA_TRY(cudaMemsetAsync(c->fb.spatial[f], 0, c->g.spatial_size() * sizeof(float), c->st));
}

static int run_move(spx_ctx* c, int s0, int s1, bool push) {
  FieldPtrs fp = field_ptrs(c);
  int launches = 0;
  if (c->plain) {
    for (int s = s0; s < s1; ++s) {
      if (push) launches += plain_push(c->species[s], c->species[s].n, c->pg, c->pp, fp, c->d_err, c->st);
      launches += plain_move_deposit(c->species[s], c->species[s].n, c->pg, c->pp, fp, c->d_err, c->st);
    }
    return launches;
  }
  return slot_step(c->species.data(), s0, s1, c->pg, c->pp, fp, push, true, c->d_err, c->st);
}

static int run_push_only(spx_ctx* c, int s0, int s1) {
  FieldPtrs fp = field_ptrs(c);
  if (c->plain) {
    int l = 0;
    for (int s = s0; s < s1; ++s) l += plain_push(c->species[s], c->species[s].n, c->pg, c->pp, fp, c->d_err, c->st);
    return l;
  }
  return slot_step(c->species.data(), s0, s1, c->pg, c->pp, fp, true, false, c->d_err, c->st);
}

static int fold_all(spx_ctx* c) {
  float* f[5] = {c->fb.spatial[SPX_JX], c->fb.spatial[SPX_JY], c->fb.spatial[SPX_JZ], c->fb.spatial[SPX_DSTY],
                 c->fb.spatial[SPX_DENS]};
  launch_fold(c->g, f, 5, c->st);
  return 1;
}

extern "C" int spx_flush(spx_ctx* c) {
  if (!c) return SPX_ERR_ARG;
  if (!c->pending_push) return SPX_OK;
  SPX_GUARD(c, {
    c->pending_push = false;
    run_push_only(c, 0, (int)c->species.size());
    return check_device_error(c);
  });
  return SPX_OK;
}

extern "C" int spx_synchronize(spx_ctx* c) {
  if (!c) return SPX_ERR_ARG;
  SPX_GUARD(c, { SPX_CUDA_TRY(cudaStreamSynchronize(c->st)); });
  return SPX_OK;
}

extern "C" int spx_zero_sources(spx_ctx* c) {
  if (!c) return SPX_ERR_ARG;
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    zero_sources(c);
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

extern "C" int spx_move_and_deposit(spx_ctx* c, int32_t s) {
  if (!c) return SPX_ERR_ARG;
  if (s < 0 || s >= (int)c->species.size()) return fail(c, SPX_ERR_ARG, "no such species");
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    run_move(c, s, s + 1, false);
    invalidate_graphs(c);
    return check_device_error(c);
  });
  return SPX_OK;
}

extern "C" int spx_boris_push(spx_ctx* c, int32_t s) {
  if (!c) return SPX_ERR_ARG;
  if (s < 0 || s >= (int)c->species.size()) return fail(c, SPX_ERR_ARG, "no such species");
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    run_push_only(c, s, s + 1);
    return check_device_error(c);
  });
  return SPX_OK;
}

extern "C" int spx_deposit_ghosts(spx_ctx* c, int32_t field) {
  if (!c) return SPX_ERR_ARG;
  if (field < 0 || field >= SPX_NUM_FIELDS) return fail(c, SPX_ERR_ARG, "no such field");
  SPX_GUARD(c, {
    float* f = c->fb.spatial[field];
    launch_fold(c->g, &f, 1, c->st);
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

extern "C" int spx_fields_update(spx_ctx* c) {
  if (!c) return SPX_ERR_ARG;
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    field_update(c->fb, c->st);
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

static void capture_steady_state(spx_ctx* c);

extern "C" int spx_prepare(spx_ctx* c) {
  if (!c) return SPX_ERR_ARG;
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    run_move(c, 0, (int)c->species.size(), false);  // src/lib.rs:130-132
    fold_all(c);                                      // src/lib.rs:134-142
    invalidate_graphs(c);
    if (int e = check_device_error(c)) return e;
    capture_steady_state(c);
  });
  return SPX_OK;
}

__global__ void k_pack_cells(uint64_t n, const uint32_t* ix, const uint32_t* iy, uint32_t* cell) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    cell[i] = ix[i] | (iy[i] << 16);
}
void pack_cells(uint64_t n, const uint32_t* ix, const uint32_t* iy, uint32_t* cell, cudaStream_t st) {
  if (n) k_pack_cells<<<148 * 8, 256, 0, st>>>(n, ix, iy, cell);
}

// Overflow handling: if a species parked particles in its overflow list,
// rebuild its slots with a larger K (the list keeps results exact meanwhile).
static void maybe_repack(spx_ctx* c) {
  if (c->plain) return;
  c->last_overflow = 0;
  c->last_max_occ = 0;
  for (auto& s : c->species) {
    SlotSpecies& S = s.slot;
    uint32_t h[2] = {0, 0};
    SPX_CUDA_TRY(cudaMemsetAsync(c->d_u32, 0, sizeof(uint32_t), c->st));
    slot_max_occupancy(s, c->pg, c->d_u32, c->st);
    SPX_CUDA_TRY(cudaMemcpyAsync(&h[0], c->d_u32, 4, cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaMemcpyAsync(&h[1], S.ocount + S.ocur, 4, cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    c->last_overflow += h[1];
    c->last_max_occ = std::max<uint64_t>(c->last_max_occ, h[0]);
    // The overflow list keeps every particle exact, but its fallback kernel is slower per
    // particle: the slots grow once it holds more than 1/256 of the species.  The capacity
    // is one number for all cells, so a few dense cells (a bunching beam, a shock) must not
    // grow every cell's slots after each overflow until the device is full: a repack whose
    // slots would not fit leaves the particles in the overflow list (its capacity, n/32,
    // is checked every step: SPX_ERR_STATE when exceeded).
    const uint64_t n = s.n;
    if ((uint64_t)h[1] <= std::max<uint64_t>(n / 256, 64)) continue;
    Capacity want = capacity_for(c, n, h[0]);
    want.KL = std::max(want.KL, S.KL + std::max(S.KL / 2, 4));
    want.H = std::max(want.H, S.H + std::max(S.H / 2, 4));
    {
      size_t free_b = 0, total_b = 0;
      SPX_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
      const double old_b = 24.0 * (double)S.ncells * S.K, new_b = 24.0 * (double)S.ncells * (want.KL + 2 * want.H);
      const double staging = 32.0 * (double)n, margin = 512.0 * 1024 * 1024;
      if (new_b + staging + margin > (double)free_b + old_b) continue;
    }
    ++c->repacks;
    // unpack (reference order) and pack again with a larger capacity
    Staging st;
    st.alloc(n);
    uint32_t *d_ix, *d_iy;
    SPX_CUDA_TRY(cudaMallocAsync(&d_ix, n * 4, c->st));
    SPX_CUDA_TRY(cudaMallocAsync(&d_iy, n * 4, c->st));
    slot_unpack(s, c->pg, d_ix, d_iy, st.dx, st.dy, st.px, st.py, st.pz, nullptr, c->pp.csqinv, c->st);
    pack_cells(n, d_ix, d_iy, st.cell, c->st);  // cell = ix | iy << 16
    slot_count(c->pg, n, st.cell, c->d_counts, c->st);
    Capacity cap = choose_capacity(c, n);
    cap.KL = std::max(cap.KL, want.KL);
    cap.H = std::max(cap.H, want.H);
    slot_release(s);
    slot_allocate(s, c->pg, cap.KL, cap.H, n);
    slot_scatter(s, c->pg, n, st.cell, st.dx, st.dy, st.px, st.py, st.pz, nullptr, c->d_counts, c->st);
    SPX_CUDA_TRY(cudaFreeAsync(d_ix, c->st));
    SPX_CUDA_TRY(cudaFreeAsync(d_iy, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    invalidate_graphs(c);
    capture_steady_state(c);
  }
}


// One loop iteration of run() in fused form.  Returns launches.
static int step_body(spx_ctx* c, bool timed, int slot) {
  int launches = 0;
  const int ns = (int)c->species.size();
  cudaEvent_t* e = timed ? &c->ev[5 * slot] : nullptr;
  if (e) SPX_CUDA_TRY(cudaEventRecord(e[4], c->st));
  zero_sources(c);  // memsets, not kernels
  if (e) SPX_CUDA_TRY(cudaEventRecord(e[0], c->st));
  if (c->plain) {
    launches += run_move(c, 0, ns, false);
  } else if (c->pending_push) {
    launches += run_move(c, 0, ns, true);  // P(t-1) fused with M(t)
  } else {
    launches += run_move(c, 0, ns, false);
  }
  if (e) SPX_CUDA_TRY(cudaEventRecord(e[1], c->st));
  launches += fold_all(c);
  if (e) SPX_CUDA_TRY(cudaEventRecord(e[2], c->st));
  launches += field_update(c->fb, c->st);
  if (c->plain) {
    launches += run_push_only(c, 0, ns);
  } else {
    c->pending_push = true;
  }
  if (e) SPX_CUDA_TRY(cudaEventRecord(e[3], c->st));
  return launches;
}

static uint32_t parity_key(spx_ctx* c) {
  uint32_t k = c->pending_push ? 1u : 0u;
  for (size_t i = 0; i < c->species.size(); ++i) k |= (uint32_t)c->species[i].slot.ocur << (i + 1);
  return k;
}

// Capturing records the work of one step without running it: the host-side
// slot state is kept as it was, and the graph is then replayed like a cached one.
static std::map<uint32_t, StepGraph>::iterator capture_step(spx_ctx* c, uint32_t key) {
  std::vector<SlotSpecies> before;
  for (auto& sp : c->species) before.push_back(sp.slot);
  cudaGraph_t gr;
  SPX_CUDA_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  const int l = step_body(c, false, 0);
  SPX_CUDA_TRY(cudaStreamEndCapture(c->st, &gr));
  cudaGraphExec_t ex;
  SPX_CUDA_TRY(cudaGraphInstantiate(&ex, gr, 0));
  SPX_CUDA_TRY(cudaGraphDestroy(gr));
  for (size_t s = 0; s < c->species.size(); ++s) c->species[s].slot = before[s];
  return c->graphs.emplace(key, StepGraph{ex, l}).first;
}

// The steady state of the split path alternates between two graphs (arrival
// region and overflow-list parity, push pending).  Capturing both up front
// keeps graph instantiation out of every later run of steps.
static void capture_steady_state(spx_ctx* c) {
  if (c->plain || !c->use_graphs || c->species.empty()) return;
  std::vector<SlotSpecies> before;
  for (auto& sp : c->species) before.push_back(sp.slot);
  const bool pend = c->pending_push;
  for (uint32_t oc = 0; oc < 2; ++oc) {
    for (auto& sp : c->species) sp.slot.ocur = oc;
    c->pending_push = true;
    const uint32_t key = parity_key(c);
    if (!c->graphs.count(key)) capture_step(c, key);
  }
  for (size_t s = 0; s < c->species.size(); ++s) c->species[s].slot = before[s];
  c->pending_push = pend;
}

extern "C" int spx_step(spx_ctx* c, uint32_t n) {
  if (!c) return SPX_ERR_ARG;
  if (c->species.empty()) return fail(c, SPX_ERR_STATE, "no species");
  SPX_GUARD(c, {
    uint64_t launches = 0;
    if (c->timing) {
      if ((int)c->ev.size() < 5 * (int)n) {
        for (auto ev : c->ev) cudaEventDestroy(ev);
        c->ev.assign(5 * n, nullptr);
        for (auto& ev : c->ev) SPX_CUDA_TRY(cudaEventCreate(&ev));
      }
      for (uint32_t i = 0; i < n; ++i) launches += step_body(c, true, (int)i);
      c->ev_steps = (int)n;
    } else if (!c->use_graphs) {
      for (uint32_t i = 0; i < n; ++i) launches += step_body(c, false, 0);
    } else {
      for (uint32_t i = 0; i < n; ++i) {
        // graphs are captured in the steady state (a push pending on the split
        // path); the first step after prepare runs uncaptured
        if (!c->plain && !c->pending_push) {
          launches += step_body(c, false, 0);
          continue;
        }
        const uint32_t key = parity_key(c);
        auto it = c->graphs.find(key);
        if (it == c->graphs.end()) it = capture_step(c, key);
        SPX_CUDA_TRY(cudaGraphLaunch(it->second.exec, c->st));
        if (!c->plain)
          for (auto& sp : c->species) sp.slot.ocur ^= 1;  // what slot_step does to the host-side state
        launches += it->second.launches;  // the kernels the graph runs
      }
    }
    c->last_launches = launches;
    if (int e = check_device_error(c)) return e;
    if (c->timing) {
      float acc[4] = {0, 0, 0, 0};
      for (int i = 0; i < c->ev_steps; ++i) {
        float a, b, d, t;
        SPX_CUDA_TRY(cudaEventElapsedTime(&a, c->ev[5 * i], c->ev[5 * i + 1]));
        SPX_CUDA_TRY(cudaEventElapsedTime(&b, c->ev[5 * i + 1], c->ev[5 * i + 2]));
        SPX_CUDA_TRY(cudaEventElapsedTime(&d, c->ev[5 * i + 2], c->ev[5 * i + 3]));
        SPX_CUDA_TRY(cudaEventElapsedTime(&t, c->ev[5 * i + 4], c->ev[5 * i + 3]));
        acc[0] += a;
        acc[1] += b;
        acc[2] += d;
        acc[3] += t;
      }
      for (int k = 0; k < 4; ++k) c->last_timing[k] = acc[k];
    }
    maybe_repack(c);
  });
  return SPX_OK;
}

extern "C" int spx_set_timing(spx_ctx* c, int32_t enable) {
  if (!c) return SPX_ERR_ARG;
  c->timing = enable != 0;
  return SPX_OK;
}
extern "C" int spx_get_timing(spx_ctx* c, float* out4) {
  if (!c || !out4) return SPX_ERR_ARG;
  for (int k = 0; k < 4; ++k) out4[k] = c->last_timing[k];
  return SPX_OK;
}
extern "C" uint64_t spx_last_launch_count(const spx_ctx* c) { return c ? c->last_launches : 0; }
extern "C" void* spx_get_stream(const spx_ctx* c) { return c ? (void*)c->st : nullptr; }
extern "C" int spx_get_counters(const spx_ctx* c, uint64_t* out8) {
  if (!c || !out8) return SPX_ERR_ARG;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  out8[0] = c->repacks;
  out8[1] = c->last_overflow;
  out8[2] = c->last_max_occ;
  out8[3] = c->species.empty() ? 0 : (uint64_t)c->species[0].slot.K;
  out8[4] = (uint64_t)c->pg.ntiles();
  out8[5] = (uint64_t)c->pg.TC();
  out8[6] = c->last_launches;
  out8[7] = (uint64_t)(total_b - free_b);
  return SPX_OK;
}

// ---------------------------------------------------------------- field access
extern "C" int spx_get_field(spx_ctx* c, int32_t field, int32_t with_ghosts, float* out) {
  if (!c || !out) return SPX_ERR_ARG;
  if (field < 0 || field >= SPX_NUM_FIELDS) return fail(c, SPX_ERR_ARG, "no such field");
  SPX_GUARD(c, {
    const float* src = c->fb.spatial[field];
    if (with_ghosts) {
      SPX_CUDA_TRY(cudaMemcpyAsync(out, src, c->g.spatial_size() * 4, cudaMemcpyDeviceToHost, c->st));
    } else {
      // interior rows (save_fld_spatial, src/save/mod.rs:14-17)
      SPX_CUDA_TRY(cudaMemcpy2DAsync(out, c->g.nx * 4, src + c->g.W + 1, c->g.W * 4, c->g.nx * 4, c->g.ny,
                                     cudaMemcpyDeviceToHost, c->st));
    }
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

extern "C" int spx_set_field(spx_ctx* c, int32_t field, const float* in) {
  if (!c || !in) return SPX_ERR_ARG;
  if (field < 0 || field >= SPX_NUM_FIELDS) return fail(c, SPX_ERR_ARG, "no such field");
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    SPX_CUDA_TRY(cudaMemcpyAsync(c->fb.spatial[field], in, c->g.spatial_size() * 4, cudaMemcpyHostToDevice, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

// B_wrk is kept as a half spectrum (kx in [0, nx/2)); the caller sees the full
// ny x nx array: kx > nx/2 from the conjugate mirror, column nx/2 zero.
extern "C" int spx_get_bwrk(spx_ctx* c, int32_t comp, float* out) {
  if (!c || !out || comp < 0 || comp > 2) return SPX_ERR_ARG;
  SPX_GUARD(c, {
    const int nx = c->g.nx, ny = c->g.ny, H = nx / 2;
    std::vector<float2> half(c->g.half_spectral_size());
    SPX_CUDA_TRY(cudaMemcpyAsync(half.data(), c->fb.spec[SP_BWX + comp], half.size() * sizeof(float2),
                                 cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    float2* o = reinterpret_cast<float2*>(out);
    for (int i = 0; i < ny; ++i)
      for (int j = 0; j < nx; ++j) {
        float2 v = make_float2(0.f, 0.f);
        if (j < H) {
          v = half[(size_t)i * H + j];
        } else if (j > H) {
          const float2 m = half[(size_t)((ny - i) & (ny - 1)) * H + (nx - j)];
          v = make_float2(m.x, -m.y);
        }
        o[(size_t)i * nx + j] = v;
      }
  });
  return SPX_OK;
}

// Keeps kx in [0, nx/2) of the caller's full array (the spectrum of a real field
// is fixed by that half).
extern "C" int spx_set_bwrk(spx_ctx* c, int32_t comp, const float* in) {
  if (!c || !in || comp < 0 || comp > 2) return SPX_ERR_ARG;
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    const int nx = c->g.nx, ny = c->g.ny, H = nx / 2;
    std::vector<float2> half(c->g.half_spectral_size());
    const float2* src = reinterpret_cast<const float2*>(in);
    for (int i = 0; i < ny; ++i)
      std::memcpy(&half[(size_t)i * H], src + (size_t)i * nx, (size_t)H * sizeof(float2));
    SPX_CUDA_TRY(cudaMemcpyAsync(c->fb.spec[SP_BWX + comp], half.data(), half.size() * sizeof(float2),
                                 cudaMemcpyHostToDevice, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
  });
  return SPX_OK;
}

// ---------------------------------------------------------------- diagnostics
__global__ void k_field_energy(const float* a, const float* b, const float* cc, Grid g, double* out) {
  double e = 0;
  const size_t n = (size_t)g.nx * g.ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / g.nx + 1, col = i % g.nx + 1;
    const size_t o = r * g.W + col;
    const double x = a[o], y = b[o], z = cc ? cc[o] : 0.0;
    e += cc ? 0.5 * (x * x + y * y + z * z) : x;
  }
  for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, e);
}

extern "C" int spx_diag(spx_ctx* c, double* out5) {
  if (!c || !out5) return SPX_ERR_ARG;
  SPX_GUARD(c, {
    if (int e = spx_flush(c)) return e;
    SPX_CUDA_TRY(cudaMemsetAsync(c->d_diag, 0, 8 * sizeof(double), c->st));
    k_field_energy<<<148 * 4, 256, 0, c->st>>>(c->fb.spatial[SPX_EX], c->fb.spatial[SPX_EY], c->fb.spatial[SPX_EZ],
                                                c->g, c->d_diag + 0);
    k_field_energy<<<148 * 4, 256, 0, c->st>>>(c->fb.spatial[SPX_BX], c->fb.spatial[SPX_BY], c->fb.spatial[SPX_BZ],
                                                c->g, c->d_diag + 1);
    for (auto& s : c->species) kinetic_energy(s, c->pg, c->plain, c->prm.c, c->d_diag + 2, c->st);
    // net charge: interior sum of dsty (the third pointer null -> plain sum)
    k_field_energy<<<148 * 4, 256, 0, c->st>>>(c->fb.spatial[SPX_DSTY], nullptr, nullptr, c->g, c->d_diag + 4);
    double h[8];
    SPX_CUDA_TRY(cudaMemcpyAsync(h, c->d_diag, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    SPX_CUDA_TRY(cudaStreamSynchronize(c->st));
    out5[0] = h[0];
    out5[1] = h[1];
    out5[2] = h[2];
    out5[3] = h[4];
    out5[4] = h[3];
  });
  return SPX_OK;
}

// ---------------------------------------------------------------- standalone ops
extern "C" int spx_field_op(uint64_t nx, uint64_t ny, int32_t op, uint32_t n_pass, float* spatial) {
  if (!spatial || nx < 2 || ny < 2 || op < 0 || op > 3) return fail(nullptr, SPX_ERR_ARG, "bad field op arguments");
  if (op == 3 && !filter_fused_fits(n_pass)) return fail(nullptr, SPX_ERR_ARG, "n_pass out of the fused filter's range");
  try {
    Grid g{(int)nx, (int)ny, (int)nx + 2, 0, 0};
    const size_t bytes = g.spatial_size() * 4;
    float *a = nullptr, *b = nullptr;
    SPX_CUDA_TRY(cudaMalloc(&a, bytes));
    SPX_CUDA_TRY(cudaMalloc(&b, bytes));
    SPX_CUDA_TRY(cudaMemcpy(a, spatial, bytes, cudaMemcpyHostToDevice));
    if (op == 0) launch_fold(g, &a, 1, 0);
    else if (op == 1) launch_update_ghosts(g, &a, 1, 0);
    else if (op == 3) {  // the fused kernel of Flds::update, then the ghost fill its consumer does
      fields_set_kernel_attributes();
      launch_filter_fused(g, &a, &b, 1, n_pass, 0);
      launch_update_ghosts(g, &b, 1, 0);
      std::swap(a, b);
    } else {
      for (uint32_t p = 0; p < n_pass; ++p) {
        launch_filter_pass(g, &a, &b, 1, 0);
        std::swap(a, b);
      }
    }
    SPX_CUDA_TRY(cudaGetLastError());
    SPX_CUDA_TRY(cudaMemcpy(spatial, a, bytes, cudaMemcpyDeviceToHost));
    cudaFree(a);
    cudaFree(b);
  } catch (const spx::Error& e) {
    return fail(nullptr, e.code, e.msg);
  }
  return SPX_OK;
}

extern "C" int spx_fft2d(uint64_t nx, uint64_t ny, int32_t inverse, float* data) {
  if (!data || !is_pow2(nx) || !is_pow2(ny) || nx < 8 || ny < 8 || nx > 8192 || ny > 8192)
    return fail(nullptr, SPX_ERR_ARG, "GPU FFT needs power-of-two sizes in [8, 8192]");
  try {
    Grid g{(int)nx, (int)ny, (int)nx + 2, ilog2(nx), ilog2(ny)};
    const size_t bytes = nx * ny * 8;
    float2* d = nullptr;
    float2 *tx = nullptr, *ty = nullptr;
    SPX_CUDA_TRY(cudaMalloc(&d, bytes));
    const std::vector<float2> twx = make_pass_twiddles((int)nx), twy = make_pass_twiddles((int)ny);
    SPX_CUDA_TRY(cudaMalloc(&tx, twx.size() * 8));
    SPX_CUDA_TRY(cudaMalloc(&ty, twy.size() * 8));
    SPX_CUDA_TRY(cudaMemcpy(tx, twx.data(), twx.size() * 8, cudaMemcpyHostToDevice));
    SPX_CUDA_TRY(cudaMemcpy(ty, twy.data(), twy.size() * 8, cudaMemcpyHostToDevice));
    SPX_CUDA_TRY(cudaMemcpy(d, data, bytes, cudaMemcpyHostToDevice));
    fields_set_kernel_attributes();
    fft2d_inplace(g, d, tx, ty, inverse != 0, 0);
    SPX_CUDA_TRY(cudaMemcpy(data, d, bytes, cudaMemcpyDeviceToHost));
    cudaFree(d);
    cudaFree(tx);
    cudaFree(ty);
  } catch (const spx::Error& e) {
    return fail(nullptr, e.code, e.msg);
  }
  return SPX_OK;
}

// ======================================================================
// Batches of independent simulations (uneven grids and particle counts).
// The particle phase of every simulation is one persistent launch over a
// work queue of (simulation, tile) items; the field phase of each simulation
// runs on its own stream; one step of the whole batch is one CUDA graph.
// ======================================================================
struct spx_batch {
  std::vector<spx_ctx*> sims;
  cudaStream_t st = nullptr;
  SlotBatch sb;
  FieldBatch* fbat = nullptr;  // the members' field phase, grouped by grid
  UploadRing up;  // one upload ring lent to every member (they add species one after another)
  bool built = false;
  std::map<uint32_t, StepGraph> graphs;
  std::string err;
  bool timing = false;
  cudaEvent_t t0 = nullptr, tz = nullptr, t1 = nullptr, t2 = nullptr;  // step start, sources zeroed, particles, end
  float last_ms[2] = {0, 0};  // particle phase, whole step (summed over the last call)
  uint64_t last_launches = 0;
};

static int bfail(spx_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  else g_create_err = m;
  return code;
}

static std::vector<SlotBatchSim> batch_sims(spx_batch* b) {
  std::vector<SlotBatchSim> v;
  for (spx_ctx* c : b->sims) {
    SlotBatchSim m;
    m.sp = c->species.data();
    m.ns = (int)c->species.size();
    m.pg = c->pg;
    m.pp = c->pp;
    m.fp = field_ptrs(c);
    m.derr = c->d_err;
    v.push_back(m);
  }
  return v;
}

extern "C" int spx_batch_create(int32_t n, const spx_params* params, spx_batch** out) {
  if (!out || !params || n <= 0) return bfail(nullptr, SPX_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  spx_batch* b = new spx_batch();
  try {
    for (int i = 0; i < n; ++i) {
      spx_params p = params[i];
      if (p.path == SPX_PATH_PLAIN) throw spx::Error(SPX_ERR_ARG, "a batch runs the split path");
      if (p.compensated) throw spx::Error(SPX_ERR_ARG, "compensated currents are a single-simulation option");
      // one tile shape for the whole batch: 8 x 8 (measured on the 64-shock ensemble: 3 % faster
      // than 16 x 16; smaller CTAs wait less for their slowest warp at the tile's barriers)
      if (p.tile_x <= 0 && p.tile_y <= 0) p.tile_x = p.tile_y = 8;
      spx_ctx* c = nullptr;
      int rc = spx_create(&p, &c);
      if (rc) throw spx::Error(rc, std::string("simulation ") + std::to_string(i) + ": " + g_create_err);
      c->use_graphs = false;  // members advance through the batch's own graphs
      c->up = &b->up;
      b->sims.push_back(c);
      if (c->pg.TX != b->sims[0]->pg.TX || c->pg.TY != b->sims[0]->pg.TY)
        throw spx::Error(SPX_ERR_ARG, "all simulations of a batch need the same tile shape");
    }
    SPX_CUDA_TRY(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    SPX_CUDA_TRY(cudaEventCreate(&b->t0));
    SPX_CUDA_TRY(cudaEventCreate(&b->tz));
    SPX_CUDA_TRY(cudaEventCreate(&b->t1));
    SPX_CUDA_TRY(cudaEventCreate(&b->t2));
  } catch (const spx::Error& e) {
    spx_batch_destroy(b);
    return bfail(nullptr, e.code, e.msg);
  }
  *out = b;
  return SPX_OK;
}

extern "C" int spx_batch_destroy(spx_batch* b) {
  if (!b) return SPX_OK;
  if (b->st) cudaStreamSynchronize(b->st);
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.exec);
  b->sb.release();
  field_batch_release(b->fbat);
  b->fbat = nullptr;
  for (spx_ctx* c : b->sims) spx_destroy(c);
  b->up.release();
  for (auto e : {b->t0, b->tz, b->t1, b->t2})
    if (e) cudaEventDestroy(e);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return SPX_OK;
}

extern "C" const char* spx_batch_last_error(const spx_batch* b) { return b ? b->err.c_str() : g_create_err.c_str(); }

extern "C" spx_ctx* spx_batch_sim(spx_batch* b, int32_t i) {
  if (!b || i < 0 || i >= (int)b->sims.size()) return nullptr;
  return b->sims[i];
}

static void capture_batch_steady_state(spx_batch* b);

extern "C" int spx_batch_prepare(spx_batch* b) {
  if (!b) return SPX_ERR_ARG;
  if (cudaSetDevice(b->sims[0]->prm.device) != cudaSuccess) return bfail(b, SPX_ERR_CUDA, "cudaSetDevice failed");
  for (size_t i = 0; i < b->sims.size(); ++i) {
    spx_ctx* c = b->sims[i];
    if (c->species.empty()) return bfail(b, SPX_ERR_STATE, "simulation " + std::to_string(i) + " has no species");
    if (int rc = spx_prepare(c)) return bfail(b, rc, "simulation " + std::to_string(i) + ": " + c->err);
  }
  // The members' shared upload scratch stays until spx_batch_destroy (~0.2 GB plus
  // 4 B per particle of the largest species): releasing device memory here took up
  // to 0.7 s on some devices, inside the caller's set-up.
  try {
    b->sb.release();
    slot_batch_build(b->sb, batch_sims(b));
    field_batch_release(b->fbat);
    b->fbat = nullptr;
    std::vector<FieldBuffers*> fbs;
    for (spx_ctx* c : b->sims) fbs.push_back(&c->fb);
    b->fbat = field_batch_build(fbs);
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.exec);
    b->graphs.clear();
    capture_batch_steady_state(b);
    b->built = true;
  } catch (const spx::Error& e) {
    return bfail(b, e.code, e.msg);
  }
  return SPX_OK;
}

// One step of every simulation.  Returns kernel launches.
// The sources of every member are zeroed and, after the particle phase, folded
// and advanced by the batched field phase (one launch per kernel and grid group).
static int batch_step_body(spx_batch* b, bool timed) {
  int launches = 0;
  if (timed) SPX_CUDA_TRY(cudaEventRecord(b->t0, b->st));
  launches += field_batch_zero_sources(b->fbat, b->st);
  if (timed) SPX_CUDA_TRY(cudaEventRecord(b->tz, b->st));
  std::vector<SlotBatchSim> sims = batch_sims(b);
  const bool pending = b->sims[0]->pending_push;
  launches += slot_batch_step(b->sb, sims, pending, true, b->st);
  if (timed) SPX_CUDA_TRY(cudaEventRecord(b->t1, b->st));
  launches += field_batch_update(b->fbat, b->st);
  for (spx_ctx* c : b->sims) c->pending_push = true;
  if (timed) SPX_CUDA_TRY(cudaEventRecord(b->t2, b->st));
  return launches;
}

static uint32_t batch_key(spx_batch* b) {
  return (uint32_t)b->sims[0]->species[0].slot.ocur | ((uint32_t)b->sims[0]->pending_push << 1);
}

// As capture_step, for one step of the whole batch.
static std::map<uint32_t, StepGraph>::iterator capture_batch_step(spx_batch* b, uint32_t key) {
  std::vector<std::vector<SlotSpecies>> before;
  std::vector<bool> pend;
  for (spx_ctx* c : b->sims) {
    std::vector<SlotSpecies> v;
    for (auto& sp : c->species) v.push_back(sp.slot);
    before.push_back(v);
    pend.push_back(c->pending_push);
  }
  cudaGraph_t gr;
  SPX_CUDA_TRY(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  const int l = batch_step_body(b, false);
  SPX_CUDA_TRY(cudaStreamEndCapture(b->st, &gr));
  cudaGraphExec_t ex;
  SPX_CUDA_TRY(cudaGraphInstantiate(&ex, gr, 0));
  SPX_CUDA_TRY(cudaGraphDestroy(gr));
  for (size_t i = 0; i < b->sims.size(); ++i) {
    for (size_t s = 0; s < b->sims[i]->species.size(); ++s) b->sims[i]->species[s].slot = before[i][s];
    b->sims[i]->pending_push = pend[i];
  }
  return b->graphs.emplace(key, StepGraph{ex, l}).first;
}

// As capture_steady_state: the four graphs of the batch's steady state.
static void capture_batch_steady_state(spx_batch* b) {
  std::vector<std::vector<SlotSpecies>> before;
  std::vector<bool> pend;
  for (spx_ctx* c : b->sims) {
    std::vector<SlotSpecies> v;
    for (auto& sp : c->species) v.push_back(sp.slot);
    before.push_back(v);
    pend.push_back(c->pending_push);
  }
  for (uint32_t oc = 0; oc < 2; ++oc) {
    for (spx_ctx* c : b->sims) {
      for (auto& sp : c->species) sp.slot.ocur = oc;
      c->pending_push = true;
    }
    const uint32_t key = batch_key(b);
    if (!b->graphs.count(key)) capture_batch_step(b, key);
  }
  for (size_t i = 0; i < b->sims.size(); ++i) {
    for (size_t s = 0; s < b->sims[i]->species.size(); ++s) b->sims[i]->species[s].slot = before[i][s];
    b->sims[i]->pending_push = pend[i];
  }
}

extern "C" int spx_batch_step(spx_batch* b, uint32_t steps) {
  if (!b) return SPX_ERR_ARG;
  if (cudaSetDevice(b->sims[0]->prm.device) != cudaSuccess) return bfail(b, SPX_ERR_CUDA, "cudaSetDevice failed");
  if (!b->built) return bfail(b, SPX_ERR_STATE, "spx_batch_prepare first");
  try {
    // the batch advances in lock-step: same region parity and pending push
    for (spx_ctx* c : b->sims)
      for (auto& sp : c->species)
        if (sp.slot.ocur != b->sims[0]->species[0].slot.ocur || c->pending_push != b->sims[0]->pending_push)
          return bfail(b, SPX_ERR_STATE, "simulations of the batch were stepped separately");
    uint64_t launches = 0;
    float acc[2] = {0, 0};
    for (uint32_t k = 0; k < steps; ++k) {
      if (b->timing) {
        launches += batch_step_body(b, true);
        SPX_CUDA_TRY(cudaEventSynchronize(b->t2));
        float p = 0, t = 0;
        SPX_CUDA_TRY(cudaEventElapsedTime(&p, b->tz, b->t1));
        SPX_CUDA_TRY(cudaEventElapsedTime(&t, b->t0, b->t2));
        acc[0] += p;
        acc[1] += t;
        continue;
      }
      const uint32_t key = batch_key(b);
      auto it = b->graphs.find(key);
      if (it == b->graphs.end()) it = capture_batch_step(b, key);
      SPX_CUDA_TRY(cudaGraphLaunch(it->second.exec, b->st));
      launches += it->second.launches;  // the kernels the graph runs
      // what the captured step does to the host-side state
      for (spx_ctx* c : b->sims) {
        for (auto& sp : c->species) sp.slot.ocur ^= 1;
        c->pending_push = true;
      }
    }
    SPX_CUDA_TRY(cudaStreamSynchronize(b->st));
    b->last_launches = launches;
    if (b->timing) {
      b->last_ms[0] = acc[0];
      b->last_ms[1] = acc[1];
    }
    bool repacked = false;
    for (size_t i = 0; i < b->sims.size(); ++i) {
      spx_ctx* c = b->sims[i];
      if (int rc = check_device_error(c)) return bfail(b, rc, "simulation " + std::to_string(i) + ": " + c->err);
      const uint64_t before = c->repacks;
      maybe_repack(c);
      repacked |= c->repacks != before;
    }
    if (repacked) {  // slot arrays moved: new argument tables, new graphs
      for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.exec);
      b->graphs.clear();
      b->sb.release();
      slot_batch_build(b->sb, batch_sims(b));
      capture_batch_steady_state(b);
    }
  } catch (const spx::Error& e) {
    return bfail(b, e.code, e.msg);
  }
  return SPX_OK;
}

extern "C" int spx_batch_set_timing(spx_batch* b, int32_t enable) {
  if (!b) return SPX_ERR_ARG;
  b->timing = enable != 0;
  return SPX_OK;
}

extern "C" int spx_batch_get_timing(spx_batch* b, float* out2) {
  if (!b || !out2) return SPX_ERR_ARG;
  out2[0] = b->last_ms[0];
  out2[1] = b->last_ms[1];
  return SPX_OK;
}

extern "C" int spx_batch_get_field(spx_batch* b, int32_t field, int32_t with_ghosts, float* const* out) {
  if (!b || !out) return SPX_ERR_ARG;
  if (field < 0 || field >= SPX_NUM_FIELDS) return bfail(b, SPX_ERR_ARG, "no such field");
  for (size_t i = 0; i < b->sims.size(); ++i)
    if (!out[i]) return bfail(b, SPX_ERR_ARG, "null output for simulation " + std::to_string(i));
  try {
    SPX_CUDA_TRY(cudaSetDevice(b->sims[0]->prm.device));
    // every member's copy queued on the batch stream, one synchronisation for all
    for (size_t i = 0; i < b->sims.size(); ++i) {
      spx_ctx* c = b->sims[i];
      SPX_CUDA_TRY(cudaStreamSynchronize(c->st));  // work queued on the member's own stream
      const float* src = c->fb.spatial[field];
      if (with_ghosts)
        SPX_CUDA_TRY(cudaMemcpyAsync(out[i], src, c->g.spatial_size() * 4, cudaMemcpyDeviceToHost, b->st));
      else  // interior rows (save_fld_spatial, src/save/mod.rs:14-17)
        SPX_CUDA_TRY(cudaMemcpy2DAsync(out[i], c->g.nx * 4, src + c->g.W + 1, c->g.W * 4, c->g.nx * 4, c->g.ny,
                                       cudaMemcpyDeviceToHost, b->st));
    }
    SPX_CUDA_TRY(cudaStreamSynchronize(b->st));
  } catch (const spx::Error& e) {
    return bfail(b, e.code, e.msg);
  }
  return SPX_OK;
}

extern "C" void* spx_batch_get_stream(const spx_batch* b) { return b ? (void*)b->st : nullptr; }
extern "C" uint64_t spx_batch_last_launch_count(const spx_batch* b) { return b ? b->last_launches : 0; }
