// Pseudo-spectral field solver of the B200 hot path (src/flds/* of the reference).
#pragma once
#include <vector>

#include "common.cuh"

namespace spx {

// Spectral work arrays: half spectra, ny x nx/2 float2 each (row-major, ky rows,
// kx in [0, nx/2); kx in (nx/2, nx) is the conjugate mirror, column nx/2 is zero).
enum SpecId {
  SP_JX = 0, SP_JY, SP_JZ, SP_RHO,  // forward transforms of the filtered sources
  SP_EX, SP_EY, SP_EZ,              // E(k): forward transform, updated in place
  SP_BWX, SP_BWY, SP_BWZ,           // B(k) at t+1/2, persistent (Flds::b_*_wrk)
  SP_BAX, SP_BAY, SP_BAZ,           // B(k) at t = average of old and new b_*_wrk
  SP_COUNT
};

struct FieldBuffers {
  Grid g;
  float* spatial[SPX_NUM_FIELDS] = {};  // reference layout, (ny+2) x (nx+2)
  float* filt_tmp[4] = {};              // ping-pong partners of jx, jy, jz, dsty for the filter
  float2* spec[SP_COUNT] = {};
  float2* tw_x = nullptr;               // exp(-2 pi i m / nx), FP64-generated
  float2* tw_y = nullptr;
  float dt = 0, c = 0;
  uint32_t dens = 1, n_pass = 0;

  void allocate(const Grid& grid);
  void release();
};

// Field::deposit_ghosts on `nf` fields in one launch (src/flds/field.rs:260-373).
void launch_fold(const Grid& g, float* const* fields, int nf, cudaStream_t st);
// Field::update_ghosts (src/flds/field.rs:142-257).
void launch_update_ghosts(const Grid& g, float* const* fields, int nf, cudaStream_t st);
// One binomial_filter_2_d pass (src/flds/field.rs:376-426) from src[f] into dst[f].
void launch_filter_pass(const Grid& g, float* const* src, float* const* dst, int nf, cudaStream_t st);
// The same for one field through cudaLaunchKernel: returns that launch's own
// status and leaves any earlier error of the caller's untouched.
cudaError_t launch_filter_pass_status(const Grid& g, const float* src, float* dst, cudaStream_t st);
// n_pass binomial_filter_2_d passes in one kernel, from src[f] into the
// interior of dst[f] (ghosts untouched); usable when filter_fused_fits(n_pass).
bool filter_fused_fits(uint32_t npass);
void launch_filter_fused(const Grid& g, float* const* src, float* const* dst, int nf, uint32_t npass,
                         cudaStream_t st);
// Flds::update (src/flds/mod.rs:87-309).  Returns the number of kernel launches.
int field_update(FieldBuffers& fb, cudaStream_t st);
// The field phase of a batch of simulations (one launch per kernel and group of
// members with the same grid and filter pass count; same arithmetic as
// field_update).  Built once over members whose buffers stay where they are.
struct FieldBatch;
FieldBatch* field_batch_build(const std::vector<FieldBuffers*>& members);
void field_batch_release(FieldBatch* b);
int field_batch_groups(const FieldBatch* b);
// Zero jx, jy, jz, dsty and dens of every member (before the particle phase).
int field_batch_zero_sources(FieldBatch* b, cudaStream_t st);
// Fold the ghost frames of the sources, then Flds::update, for every member;
// ordered after the work already queued on st, and st after it.  Returns launches.
int field_batch_update(FieldBatch* b, cudaStream_t st);
// Fft2D::fft / inv_fft on one complex array in place (tests).
int fft2d_inplace(const Grid& g, float2* data, const float2* tw_x, const float2* tw_y, bool inverse,
                  cudaStream_t st);
void fields_set_kernel_attributes();
// Host generation of the FP64 twiddle table exp(-2 pi i m / n), m in [0, n).
void make_twiddles(int n, float2* host_out);
// The table the transform kernels read: per pass, per butterfly group, its
// twiddles side by side (entries of make_twiddles(n)).
std::vector<float2> make_pass_twiddles(int n);
bool is_pow2(uint64_t v);
int ilog2(uint64_t v);

}  // namespace spx
