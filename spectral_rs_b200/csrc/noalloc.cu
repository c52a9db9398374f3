// Allocation-free variant of the binomial filter entry point.
//
// Some callers cannot call cudaMalloc: a host that runs the step inside its own
// stream-ordered loop where cudaMalloc/cudaFree would synchronize the device, a
// framework whose memory comes only from its own pooled allocator, or a driver
// that forbids allocation once the run has started.  spx_filter_noalloc takes
// the caller's device buffers for input and output and keeps its ping-pong
// scratch in a fixed, file-scope device array instead of allocating one.
#include <mutex>
#include <string>

#include "fields.cuh"

namespace {

// Ping-pong scratch of the filter passes: every GPU that loads the library
// holds this array until the process exits.
constexpr size_t kScratchFloats = (size_t)SPX_NOALLOC_MAX_CELLS;
static __device__ __align__(256) float g_filter_scratch[kScratchFloats];

// The array's name in host code is only a host-side stand-in; the device
// address is looked up once per device, with that device current.
constexpr int kMaxDevices = 64;
float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;
// Message of the calling thread's last failure: each host thread has its own,
// so threads that fail at the same time neither race nor see each other's text.
thread_local std::string g_noalloc_err;

int fail(const std::string& m, int code) {
  g_noalloc_err = "spx_filter_noalloc: " + m;
  return code;
}

int scratch_for_current_device(float** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(std::string("no usable current device: ") + cudaGetErrorString(e), SPX_ERR_CUDA);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    float* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_filter_scratch);
    if (e != cudaSuccess || !p) return fail(std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e), SPX_ERR_CUDA);
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return SPX_OK;
}

}  // namespace

extern "C" const char* spx_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" int spx_filter_noalloc(uint64_t size_x, uint64_t size_y, uint32_t n_pass, const float* d_in,
                                  float* d_out, void* stream) {
  // every argument check comes before the first CUDA call
  if (!d_in || !d_out || size_x < 2 || size_y < 2) return fail("null buffer or grid smaller than 2 x 2", SPX_ERR_ARG);
  // each side alone bounded first, so the product below cannot wrap
  if (size_x > SPX_NOALLOC_MAX_CELLS || size_y > SPX_NOALLOC_MAX_CELLS)
    return fail("size_x and size_y must each be at most " + std::to_string(kScratchFloats), SPX_ERR_ARG);
  const size_t cells = (size_t)(size_x + 2) * (size_t)(size_y + 2);
  if (cells > kScratchFloats)
    return fail("(size_x+2)*(size_y+2) = " + std::to_string(cells) + " exceeds the fixed scratch of " +
                    std::to_string(kScratchFloats) + " floats",
                SPX_ERR_ARG);
  // the passes read a 3x3 neighbourhood of d_in while writing: identical or disjoint buffers only
  const uintptr_t a0 = (uintptr_t)d_in, b0 = (uintptr_t)d_out, bytes = cells * sizeof(float);
  if (d_in != d_out && a0 < b0 + bytes && b0 < a0 + bytes)
    return fail("d_in and d_out overlap without being the same buffer", SPX_ERR_ARG);
  cudaStream_t st = (cudaStream_t)stream;
  if (n_pass == 0) {
    if (d_out == d_in) return SPX_OK;
    const cudaError_t e = cudaMemcpyAsync(d_out, d_in, bytes, cudaMemcpyDeviceToDevice, st);
    return e == cudaSuccess ? SPX_OK : fail(std::string("device copy failed: ") + cudaGetErrorString(e), SPX_ERR_CUDA);
  }
  float* scratch = nullptr;
  if (int rc = scratch_for_current_device(&scratch)) return rc;
  const spx::Grid g{(int)size_x, (int)size_y, (int)size_x + 2, 0, 0};
  // Passes alternate between d_out and the scratch so that the last one lands
  // in d_out.  An in-place call (d_in == d_out) starts in the scratch and, for
  // an odd pass count, copies the result back at the end.  Each launch and
  // copy reports its own status; an earlier error of the caller's is neither
  // reported nor cleared.
  const float* src = d_in;
  const bool in_place = d_in == d_out;
  bool to_out = in_place ? false : (n_pass % 2 == 1);
  for (uint32_t p = 0; p < n_pass; ++p) {
    float* dst = to_out ? d_out : scratch;
    const cudaError_t e = spx::launch_filter_pass_status(g, src, dst, st);
    if (e != cudaSuccess) return fail(std::string("launch failed: ") + cudaGetErrorString(e), SPX_ERR_CUDA);
    src = dst;
    to_out = !to_out;
  }
  if (src != d_out) {
    const cudaError_t e = cudaMemcpyAsync(d_out, src, bytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return fail(std::string("device copy failed: ") + cudaGetErrorString(e), SPX_ERR_CUDA);
  }
  return SPX_OK;
}
