/*
 * spectral_gpu.h - C ABI of the B200 per-timestep hot path of spectral_rs.
 *
 * This is the drop-in boundary.  The reference (pcrumley/spectral_rs, Rust) has
 * no FFI; its hot path is the crate-internal API that `run` (src/lib.rs:119-202)
 * calls.  Each entry point below names the reference method it replaces, so a
 * `#[cfg(feature = "gpu")]` body of that method can forward to it.
 *
 * Conventions
 *   - Every call returns an int status: 0 (SPX_OK) on success, a positive
 *     SPX_ERR_* code otherwise; spx_last_error() gives the message.  The
 *     reference panics on its asserts (e.g. src/prtls.rs:98-102,154-171); here
 *     those asserts become SPX_ERR_BOUNDS / SPX_ERR_WALL statuses.
 *   - Device memory belongs to the context.  Host pointers are caller-owned and
 *     copied; no host pointer is retained after a call returns.
 *   - One host thread and one CUDA stream per context.  Calls are ordered on
 *     that stream; getters synchronize it.
 *   - Arithmetic is FP32 (the reference's default `Float`, src/lib.rs:18-19).
 *     There is no FP64 device path and no CPU fallback inside the library.
 *   - Grid layouts are the reference's: a spatial field is row-major
 *     (size_y+2) x (size_x+2) with a one-cell ghost frame (src/flds/field.rs:57);
 *     particle cell indices include the +1 ghost offset (src/prtls.rs:206-207).
 */
#ifndef SPECTRAL_GPU_H
#define SPECTRAL_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define SPX_API __attribute__((visibility("default")))
#else
#define SPX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SPX_OK 0
#define SPX_ERR_ARG 1        /* invalid argument or unsupported size            */
#define SPX_ERR_CUDA 2       /* a CUDA runtime call failed                      */
#define SPX_ERR_BOUNDS 3     /* particle index out of the grid (ix or iy == 0)  */
#define SPX_ERR_WALL 4       /* reflecting-wall assertion (src/prtls.rs:154-171) */
#define SPX_ERR_NOMEM 5      /* device allocation failed                        */
#define SPX_ERR_STATE 6      /* call out of order (e.g. no species yet)         */
#define SPX_ERR_GAMMA 7      /* supplied Lorentz factors inconsistent with p    */
#define SPX_ERR_TIMEOUT 8    /* a bounded device wait gave up                    */

/* Field ids (the reference's Flds members, src/flds/mod.rs:15-37). */
#define SPX_EX 0
#define SPX_EY 1
#define SPX_EZ 2
#define SPX_BX 3
#define SPX_BY 4
#define SPX_BZ 5
#define SPX_JX 6
#define SPX_JY 7
#define SPX_JZ 8
#define SPX_DSTY 9 /* "Rho": charge density */
#define SPX_DENS 10 /* number density        */
#define SPX_NUM_FIELDS 11

/* Particle paths. */
#define SPX_PATH_SPLIT 0 /* integer cell + FP32 offset (the reference layout), fused, cell-ordered */
#define SPX_PATH_PLAIN 1 /* global FP32 positions x = ix + dx, per-phase kernels, global atomics    */

/* Simulation parameters.  The first block is the reference's [params] table
 * (config.toml, src/lib.rs:56-66) plus its compile-time `periodic` feature;
 * the second block is additive and defaults to 0 = automatic. */
typedef struct spx_params {
  uint64_t size_x;     /* cells in x, even (src/lib.rs:76); powers of two on the GPU FFT */
  uint64_t size_y;     /* cells in y                                                      */
  uint64_t delta;      /* wall offset (src/prtls.rs:153)                                  */
  float dt;            /* time step in 1/omega_pe                                         */
  float c;             /* speed of light in cells per 1/omega_pe                          */
  uint32_t dens;       /* particles per cell per species (normalises rho, src/flds/mod.rs:80) */
  float gamma_inj;     /* upstream Lorentz factor (init only)                             */
  uint32_t n_pass;     /* binomial filter passes per step                                 */
  int32_t periodic_x;  /* 1: periodic particles in x (cargo feature `periodic`), 0: wall  */
  int32_t left_wall;   /* 1: also reflect at ix = delta+1, mirroring the right wall; 0: the
                          reference's assertion min(ix) > delta (src/prtls.rs:163-170)     */
  /* --- B200 additions (0 = automatic) --- */
  int32_t path;        /* SPX_PATH_SPLIT or SPX_PATH_PLAIN                                */
  int32_t tile_x;      /* cells per tile in x (split path); power of two; 0: 16 (tile_y 0: 8)   */
  int32_t tile_y;      /* cells per tile in y                                              */
  int32_t slot_capacity; /* minimum particle slots per cell and species (split path);
                          negative: exactly -slot_capacity (testing the overflow path)  */
  int32_t device;      /* CUDA device ordinal                                              */
  int32_t compensated; /* 1: current sums of the split path Kahan-compensated in registers and
                          carried through the tile flush (one CTA per SM, slower); 0: plain FP32 */
  float slot_headroom; /* sort bins (split path): low-range slots per cell = headroom x the fullest
                          cell's count (at least mean + 8 sqrt(mean)), + 8; 0: 1.25 on a periodic
                          grid, 4 with a reflecting wall (a shock compresses the plasma)       */
  int32_t arrival_slots; /* slots per cell of each of the two arrival regions; 0: max(16, low/4) */
} spx_params;

typedef struct spx_ctx spx_ctx;

/* Flds::new (src/flds/mod.rs:40-65) + Sim::new (src/lib.rs:247-264). */
SPX_API int spx_create(const spx_params* params, spx_ctx** out);
SPX_API int spx_destroy(spx_ctx* ctx);
/* Message of the last failed call on ctx (or of the last failed spx_create if ctx is NULL). */
SPX_API const char* spx_last_error(const spx_ctx* ctx);
/* Static description of the library build (compile flags, arch). */
SPX_API const char* spx_version(void);

/* Prtl::new (src/prtls.rs:60-84) with caller-supplied state, in the order of
 * the Prtl fields (src/prtls.rs:8-16).  `usize` cell indices cross as uint64.
 * psa (Lorentz factors) must equal sqrt(1 + |p|^2 / c^2) as the reference keeps
 * them (src/prtls.rs:237-249,440); the GPU recomputes it and does not store it.
 * The arrays are host memory, pageable or page-locked (page-locked arrays are
 * copied at the full host-link rate, in chunks of 2^22 particles); the call
 * returns once they are no longer read.  The context keeps its upload scratch
 * (4 B per particle of the largest species added, plus 2 x 96 MB) for later
 * uploads; spx_destroy releases it (spx_batch_destroy for batch members).
 * The species id (0, 1, ...) is written to *species_out. */
SPX_API int spx_add_species(spx_ctx* ctx, float charge, float mass, float vth, uint64_t n, const uint64_t* ix,
                    const uint64_t* iy, const float* dx, const float* dy, const float* px, const float* py,
                    const float* pz, const float* psa, int32_t* species_out);

/* Seeded on-device initialisation (replaces src/prtls.rs:191-261, whose RNG is
 * unseeded): `ppc` particles per cell in columns [x0, x1) of every row,
 * positions uniform in the cell (random_positions=1) or on the reference's
 * diagonal (0); momenta Maxwellian N(0, vth*c) per component, then a drift
 * with Lorentz factor gamma_drift along sign_x*x with the Zenitani flip
 * (src/prtls.rs:240-249).  gamma_drift <= 1 means no drift. */
SPX_API int spx_init_species(spx_ctx* ctx, float charge, float mass, float vth, uint32_t ppc, uint64_t x0, uint64_t x1,
                     float gamma_drift, float sign_x, int32_t random_positions, uint64_t seed,
                     int32_t* species_out);

SPX_API uint64_t spx_species_count(const spx_ctx* ctx, int32_t species);
SPX_API int32_t spx_num_species(const spx_ctx* ctx);

/* Copy species state back in the reference's particle order.  Any pointer may
 * be NULL to skip that array.  `stride` > 1 returns every stride-th particle,
 * as save_output does (src/save/mod.rs:36-72). */
SPX_API int spx_get_species(spx_ctx* ctx, int32_t species, uint64_t stride, uint64_t* ix, uint64_t* iy, float* dx,
                    float* dy, float* px, float* py, float* pz, float* psa);

/* Prtl::tag and Prtl::track (src/prtls.rs:21-22) of one species, n entries each
 * in the reference's particle order (either pointer may be NULL to leave that
 * table as it is; track: 0 or 1 per particle).  Particles keep their reference
 * index for life, so the tables travel with them through every step at no
 * device cost.  Until set, the reference's defaults hold: tag[i] = i
 * (src/prtls.rs:213) and only particle 40 tracked (src/prtls.rs:79). */
SPX_API int spx_set_tags(spx_ctx* ctx, int32_t species, const uint64_t* tag, const uint8_t* track);
/* The same tables back, every stride-th particle (as spx_get_species). */
SPX_API int spx_get_tags(spx_ctx* ctx, int32_t species, uint64_t stride, uint64_t* tag, uint8_t* track);
/* The particle-tracking output of save_output (src/save/mod.rs:82-97) for the
 * tracked particles, in reference order, gathered on the device:
 * x = (ix + dx) / c, y = (iy + dy) / c, gamma.  *count receives the number of
 * tracked particles; with all three outputs NULL the call only counts, else
 * SPX_ERR_ARG if the count exceeds `capacity` (nothing copied).  Any output
 * pointer may be NULL. */
SPX_API int spx_get_tracked(spx_ctx* ctx, int32_t species, uint64_t capacity, float* x, float* y, float* gamma,
                            uint64_t* count);

/* Zero j_x, j_y, j_z, dsty, dens, ghosts included (src/lib.rs:157-167). */
SPX_API int spx_zero_sources(spx_ctx* ctx);
/* Sim::move_and_deposit (src/lib.rs:478-489) for one species. */
SPX_API int spx_move_and_deposit(spx_ctx* ctx, int32_t species);
/* Field::deposit_ghosts (src/flds/field.rs:260-373) on one field id. */
SPX_API int spx_deposit_ghosts(spx_ctx* ctx, int32_t field);
/* Flds::update (src/flds/mod.rs:87-309). */
SPX_API int spx_fields_update(spx_ctx* ctx);
/* Prtl::boris_push (src/prtls.rs:262-443) for one species. */
SPX_API int spx_boris_push(spx_ctx* ctx, int32_t species);

/* The pre-loop move+deposit and ghost fold of run() (src/lib.rs:130-142). */
SPX_API int spx_prepare(spx_ctx* ctx);
/* `n` iterations of run()'s loop body (src/lib.rs:151-200) without output:
 * zero sources, move_and_deposit every species, fold, Flds::update,
 * boris_push every species.  Production path: the push of step t is fused
 * with the move+deposit of step t+1 and each step is one CUDA graph launch;
 * the last push stays pending until a particle getter or a per-phase call
 * needs it, so observable state always equals the reference's. */
SPX_API int spx_step(spx_ctx* ctx, uint32_t n);
/* Complete any pending push (see spx_step). */
SPX_API int spx_flush(spx_ctx* ctx);
SPX_API int spx_synchronize(spx_ctx* ctx);

/* Field access in the reference layout: with_ghosts=1 copies (size_y+2)*(size_x+2)
 * floats, 0 copies the size_y*size_x interior (save_fld_spatial, src/save/mod.rs:8-23). */
SPX_API int spx_get_field(spx_ctx* ctx, int32_t field, int32_t with_ghosts, float* out);
/* Overwrite a spatial field (with ghosts).  Used by tests to impose fields. */
SPX_API int spx_set_field(spx_ctx* ctx, int32_t field, const float* in_with_ghosts);
/* The persistent k-space magnetic field at t+1/2 (Flds::b_*_wrk, src/flds/mod.rs:31-33),
 * size_y*size_x interleaved complex. comp 0,1,2 = x,y,z.  B is real, so its spectrum
 * is Hermitian: the library keeps kx in [0, size_x/2) (the update zeroes column
 * size_x/2).  spx_get_bwrk fills kx > size_x/2 with the conjugate mirror
 * conj(B[size_y - ky][size_x - kx]) and column size_x/2 with zeros; spx_set_bwrk
 * keeps kx in [0, size_x/2) of its input. */
SPX_API int spx_get_bwrk(spx_ctx* ctx, int32_t comp, float* out_complex);
SPX_API int spx_set_bwrk(spx_ctx* ctx, int32_t comp, const float* in_complex);

/* FP64 device diagnostics: out[0] = sum E^2/2, out[1] = sum B^2/2 (interior
 * cells), out[2] = sum over particles of m (gamma - 1) c^2, out[3] = sum of
 * the interior of dsty (net deposited charge), out[4] = particle count. */
SPX_API int spx_diag(spx_ctx* ctx, double* out5);

/* Standalone field operations on caller arrays (the reference's Field and
 * Fft2D methods, used by the known-answer tests): op 0 = deposit_ghosts,
 * 1 = update_ghosts, 2 = n_pass x binomial_filter_2_d (one kernel per pass),
 * 3 = the same through the fused n-pass kernel of spx_fields_update
 * (1 <= n_pass <= 16).  In/out in place. */
SPX_API int spx_field_op(uint64_t size_x, uint64_t size_y, int32_t op, uint32_t n_pass, float* spatial_with_ghosts);
/* Fft2D::fft / inv_fft (src/flds/fft_2d.rs:91-172) on a size_y*size_x
 * interleaved complex array, in place; inverse includes the 1/(nx*ny) scale.
 * Power-of-two sizes only. */
SPX_API int spx_fft2d(uint64_t size_x, uint64_t size_y, int32_t inverse, float* data_complex);

/* Time of the last spx_step call's work on the context stream, in ms, summed
 * over its steps: [0] particle phase (fused push + move + deposit and slot
 * relocation), [1] ghost fold, [2] Flds::update (filter + spectral solve),
 * [3] whole step.  CUDA events; filled only while timing is enabled (then the
 * steps run uncaptured, one event set per step). */
SPX_API int spx_set_timing(spx_ctx* ctx, int32_t enable);
SPX_API int spx_get_timing(spx_ctx* ctx, float* out4);
/* The context's CUDA stream (a cudaStream_t), so callers can order their own
 * work and timing events with the library's. */
SPX_API void* spx_get_stream(const spx_ctx* ctx);
/* Layout and overflow counters: out8[0] slot repacks so far, [1] particles in
 * overflow lists at the last check, [2] largest cell occupancy at the last
 * check, [3] slot capacity K of species 0, [4] tiles, [5] cells per tile,
 * [6] kernel launches of the last spx_step call, [7] device memory in use (total - free:
 * every context on the device). */
SPX_API int spx_get_counters(const spx_ctx* ctx, uint64_t* out8);
/* Number of kernel launches issued by the last spx_step call (the kernels of a
 * step launched as a CUDA graph counted one by one). */
SPX_API uint64_t spx_last_launch_count(const spx_ctx* ctx);

/* ---- Batches of independent simulations ------------------------------------
 * Many simulations with their own grids, species and parameters (uneven
 * ensembles, e.g. parameter scans of shocks) advance together: the particle phase of
 * all of them is one persistent kernel over a work queue of (simulation, tile)
 * items ordered by decreasing work, the field phase is one launch per kernel
 * for each group of simulations that share a grid and filter pass count (each
 * member's fields bit-identical to its own spx_fields_update), and one step of
 * the batch is one CUDA graph launch.  There is no
 * counterpart in the reference (one simulation per process).
 * spx_batch_sim returns the context of simulation i, used as any spx_ctx for
 * species set-up (spx_add_species / spx_init_species) and for getters; after
 * spx_batch_prepare the simulations must only be stepped through the batch.
 * All simulations use the same tile shape (8 x 8 unless params set one). */
typedef struct spx_batch spx_batch;
SPX_API int spx_batch_create(int32_t n_sims, const spx_params* params, spx_batch** out);
SPX_API int spx_batch_destroy(spx_batch* batch);
SPX_API const char* spx_batch_last_error(const spx_batch* batch);
SPX_API spx_ctx* spx_batch_sim(spx_batch* batch, int32_t sim);
SPX_API int spx_batch_prepare(spx_batch* batch);
SPX_API int spx_batch_step(spx_batch* batch, uint32_t n);
/* Timing (CUDA events, uncaptured steps when enabled): out2[0] particle phase
 * (from the zeroed sources to the deposited ones: the work-queue reset, the
 * particle kernel and its overflow fallback), out2[1] whole steps, ms summed
 * over the last spx_batch_step call. */
SPX_API int spx_batch_set_timing(spx_batch* batch, int32_t enable);
SPX_API int spx_batch_get_timing(spx_batch* batch, float* out2);
/* Field `field` of every simulation of the batch, out[i] for simulation i (each
 * laid out as spx_get_field's output), queued together and synchronised once
 * (spx_get_field per simulation synchronises per call).  Page-locked outputs
 * let the copies run back to back. */
SPX_API int spx_batch_get_field(spx_batch* batch, int32_t field, int32_t with_ghosts, float* const* out);
SPX_API void* spx_batch_get_stream(const spx_batch* batch);
/* Kernels launched by the last spx_batch_step call (inside its graphs, one by one). */
SPX_API uint64_t spx_batch_last_launch_count(const spx_batch* batch);

/* Allocation-free binomial filter, for callers that cannot call cudaMalloc:
 * a host loop that must not synchronize the device (cudaMalloc/cudaFree do),
 * a framework that hands out memory only from its own pool, or a driver that
 * forbids allocation once the run has started.  It has no counterpart in the
 * reference; it computes what spx_field_op(op = 2) computes (n_pass passes of
 * Field::binomial_filter_2_d) on device buffers the caller owns.
 *   d_in, d_out: device pointers to (size_y+2)*(size_x+2) floats.  They must be
 *   the same buffer (in place) or not overlap at all: the passes read a 3x3
 *   neighbourhood while writing, so partly overlapping buffers are rejected
 *   with SPX_ERR_ARG.  stream: a cudaStream_t (NULL = default stream).
 * The ping-pong scratch is a fixed device array of SPX_NOALLOC_MAX_CELLS floats
 * (16 MiB) that every GPU loading the library holds until exit; grids with
 * (size_x+2)*(size_y+2) above that, or either side above SPX_NOALLOC_MAX_CELLS,
 * are rejected with SPX_ERR_ARG before any CUDA call.  The first call on a
 * device looks the array's address up (cudaGetSymbolAddress), so make it before
 * any stream capture.  All calls share the one array: calls that overlap on the
 * GPU race, so order them on one stream.  The scratch is fully overwritten by
 * every pass; nothing in it needs clearing.  Each launch's own status is
 * checked; an earlier, unrelated error of the caller's is neither reported nor
 * cleared.  spx_noalloc_last_error() returns the message of the calling host
 * thread's last failed call (one message per thread). */
#define SPX_NOALLOC_MAX_CELLS (4u * 1024u * 1024u)
SPX_API int spx_filter_noalloc(uint64_t size_x, uint64_t size_y, uint32_t n_pass, const float* d_in, float* d_out,
                               void* stream);
SPX_API const char* spx_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SPECTRAL_GPU_H */
