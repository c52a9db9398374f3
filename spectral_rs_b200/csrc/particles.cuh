// Particle species storage and kernels of the B200 hot path (src/prtls.rs and
// the deposition half of src/lib.rs in the reference).
#pragma once
#include <vector>

#include "common.cuh"

namespace spx {

constexpr int MAX_SPECIES = 4;

// Split-path ("cell-slot") storage of one species.
//
// The grid is cut into tiles of TX x TY cells; tile t owns the contiguous
// block [t*K*TC, (t+1)*K*TC) of every particle array (TC = TX*TY), laid out
// slot-major: slot s of cell c (c = cell within the tile) is element
// t*K*TC + s*TC + c.  A particle's cell is implied by where it is stored, so
// a particle is {dx, dy, px, py, pz, tag} = 24 bytes (tag = its index in the
// reference's particle order, used only to return data in that order).
//
// The K = KL + 2H slots of a cell hold a low range [0, nlow) and two arrival
// regions of H slots, region r = [KL + r*H, KL + (r+1)*H) with narr[r] entries.
// A moving step with parity q (= ocur) reads the low range and region q (the
// previous step's arrivals); the thread that owns the cell writes the
// particles that stay, in order, to [0, w) (w never passes the slot being
// read), so the low range stays dense: no holes, no compaction pass.  A
// particle that leaves goes to region q^1 of its destination (slot from an
// atomic arrivals counter, bounded by H); region q is then empty.  A particle
// that finds no room (low range or region full) goes to the overflow list,
// which a fallback kernel processes every step until the host repacks with a
// larger capacity.
struct SlotSpecies {
  float* dx = nullptr;
  float* dy = nullptr;
  float* px = nullptr;
  float* py = nullptr;
  float* pz = nullptr;
  uint32_t* tag = nullptr;
  uint32_t* nlow = nullptr;  // low range extent per cell
  uint32_t* narr = nullptr;  // [2][ncells] entries of the two arrival regions
  // overflow lists (double buffered): cell packed as ix | iy << 16 (reference coords)
  uint32_t* ocell[2] = {};
  float* odx[2] = {};
  float* ody[2] = {};
  float* opx[2] = {};
  float* opy[2] = {};
  float* opz[2] = {};
  uint32_t* otag[2] = {};
  uint32_t* ocount = nullptr;  // [2]
  uint32_t ocap = 0;
  int K = 0, KL = 0, H = 0;
  size_t ncells = 0;
  void* block = nullptr;  // the one device allocation every array above is carved from
  int ocur = 0;  // arrival region and overflow list read by the next step
};

// Plain-path storage: global FP32 positions x = ix + dx, y = iy + dy in the
// reference's particle order.
struct PlainSpecies {
  float *x = nullptr, *y = nullptr, *px = nullptr, *py = nullptr, *pz = nullptr;
};

struct Species {
  float charge = 0, mass = 1, vth = 0, alpha = 0, beta = 0;
  uint64_t n = 0;
  SlotSpecies slot;
  PlainSpecies plain;
};

struct ParticleGeom {
  Grid g;
  int TX = 16, TY = 16, logTX = 4, logTY = 4, NTX = 1, NTY = 1;
  int TC() const { return TX * TY; }
  int ntiles() const { return NTX * NTY; }
  size_t ncells() const { return (size_t)g.nx * g.ny; }
};

struct PhysParams {
  float dt, c, csqinv;
  int periodic_x, left_wall, wall_loc, delta;
  int compensated;  // compensated (Kahan) current sums in the split-path kernel
};

struct FieldPtrs {
  const float* E[3];
  const float* B[3];
  float* J[3];
  float* dsty;
  float* dens;
};

// Device error word bits.
enum : int { DERR_BOUNDS = 1, DERR_WALL = 2, DERR_OVERFLOW_LOST = 4, DERR_GAMMA = 8, DERR_TIMEOUT = 16 };

// --- split path ---------------------------------------------------------------
// Storage for n particles with a low range of KL slots and arrival regions of
// H slots per cell (its counters are set by slot_scatter_end).
void slot_allocate(Species& s, const ParticleGeom& pg, int KL, int H, uint64_t n);
void slot_release(Species& s);
// Count particles per cell (for choosing K).  counts: ncells uint32, zeroed
// first unless reset is false (a later chunk of the same species).
void slot_count(const ParticleGeom& pg, uint64_t n, const uint32_t* cell, uint32_t* counts, cudaStream_t st,
                bool reset = true);
// Place n particles into the slots allocated by slot_allocate (tags: tag[i],
// or i when tag is null).  cursor: ncells uint32 scratch.
void slot_scatter(Species& s, const ParticleGeom& pg, uint64_t n, const uint32_t* cell, const float* dx,
                  const float* dy, const float* px, const float* py, const float* pz, const uint32_t* tag,
                  uint32_t* cursor, cudaStream_t st);
// The same in chunks: begin, then chunks of the species in any order (the
// chunk's particles get tags tag0 + i when tag is null), then end.
void slot_scatter_begin(Species& s, const ParticleGeom& pg, uint32_t* cursor, cudaStream_t st);
void slot_scatter_chunk(Species& s, const ParticleGeom& pg, uint64_t n, uint32_t tag0, const uint32_t* cell,
                        const float* dx, const float* dy, const float* px, const float* py, const float* pz,
                        const uint32_t* tag, uint32_t* cursor, cudaStream_t st);
void slot_scatter_end(Species& s, const ParticleGeom& pg, uint32_t* cursor, cudaStream_t st);
// Download in reference order into device arrays indexed by tag.
void slot_unpack(const Species& s, const ParticleGeom& pg, uint32_t* ix, uint32_t* iy, float* dx, float* dy,
                 float* px, float* py, float* pz, float* psa, float csqinv, cudaStream_t st);
// The fused particle kernel over species [s0, s1): PUSH = Boris push
// (src/prtls.rs:262-443), MOVE = move_and_deposit (src/lib.rs:478-489) with
// relocation.  Returns the number of kernel launches (memsets not counted).
int slot_step(Species* sp, int s0, int s1, const ParticleGeom& pg, const PhysParams& pp, const FieldPtrs& fp,
              bool push, bool move, int* derr, cudaStream_t st);
// Maximum cell occupancy (low range + pending arrivals), reported with the layout counters.
void slot_set_kernel_attributes();
void slot_max_occupancy(const Species& s, const ParticleGeom& pg, uint32_t* d_out, cudaStream_t st);

// --- batches of simulations (one persistent launch over a work queue) -----------
struct StepArgs;
struct SlotBatchSim {
  Species* sp;  // the simulation's species array
  int ns;
  ParticleGeom pg;
  PhysParams pp;
  FieldPtrs fp;
  int* derr;
};
struct SlotBatch {
  StepArgs* d_args[2] = {nullptr, nullptr};  // per overflow-list parity
  int2* d_items = nullptr;                   // (simulation, tile), heaviest first
  int nitems = 0, nsims = 0, grid = 0;
  int* d_counter = nullptr;
  void release();
};
// Build the work list and argument tables (again after any repack).  All
// simulations must share the tile shape.
void slot_batch_build(SlotBatch& b, const std::vector<SlotBatchSim>& sims);
// One particle phase for every simulation: reset, persistent particle kernel,
// overflow fallback.  Advances the host-side slot state.  Returns kernel launches.
int slot_batch_step(SlotBatch& b, std::vector<SlotBatchSim>& sims, bool push, bool move, cudaStream_t st);

// --- plain path ---------------------------------------------------------------
int plain_move_deposit(Species& s, uint64_t n, const ParticleGeom& pg, const PhysParams& pp, const FieldPtrs& fp,
                       int* derr, cudaStream_t st);
int plain_push(Species& s, uint64_t n, const ParticleGeom& pg, const PhysParams& pp, const FieldPtrs& fp,
               int* derr, cudaStream_t st);

// The tracking output of src/save/mod.rs:85-97 for the particles with
// rank[reference index] >= 0: x = (ix + dx) / c, y = (iy + dy) / c, gamma, each
// written at that rank.
void gather_tracked(const Species& s, const ParticleGeom& pg, bool plain, const int32_t* rank, float c, float* x,
                    float* y, float* g, cudaStream_t st);

// --- diagnostics ----------------------------------------------------------------
// Adds sum m (gamma-1) c^2 and the particle count into d_acc[0], d_acc[1] (double).
void kinetic_energy(const Species& s, const ParticleGeom& pg, bool plain, float c, double* d_acc, cudaStream_t st);

// --- device initialisation (seeded) ----------------------------------------------
struct InitSpec {
  float charge, mass, vth, gamma_drift, sign_x, c;
  uint32_t ppc;
  int x0, x1;  // columns [x0, x1) of the interior (0-based), every row
  int random_positions;
  uint64_t seed;
};
// Writes particles [off, off + n) of the species, in the reference's particle
// order, into device arrays (cell packed, dx, dy, px, py, pz) indexed from 0;
// particle i depends only on i and the seed, so any chunking gives the same species.
void init_particles(const InitSpec& is, const Grid& g, uint64_t off, uint64_t n, uint32_t* cell, float* dx,
                    float* dy, float* px, float* py, float* pz, cudaStream_t st);

}  // namespace spx
