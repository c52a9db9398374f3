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
std::string g_noalloc_err;

int scratch_for_current_device(float** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    g_noalloc_err = std::string("spx_filter_noalloc: no usable current device: ") + cudaGetErrorString(e);
    return SPX_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    float* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_filter_scratch);
    if (e != cudaSuccess || !p) {
      g_noalloc_err = std::string("spx_filter_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return SPX_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return SPX_OK;
}

}  // namespace

extern "C" const char* spx_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" int spx_filter_noalloc(uint64_t size_x, uint64_t size_y, uint32_t n_pass, const float* d_in,
                                  float* d_out, void* stream) {
  if (!d_in || !d_out || size_x < 2 || size_y < 2) {
    g_noalloc_err = "spx_filter_noalloc: null buffer or grid smaller than 2 x 2";
    return SPX_ERR_ARG;
  }
  const size_t cells = (size_t)(size_x + 2) * (size_t)(size_y + 2);
  if (cells > kScratchFloats) {
    g_noalloc_err = "spx_filter_noalloc: (size_x+2)*(size_y+2) = " + std::to_string(cells) +
                    " exceeds the fixed scratch of " + std::to_string(kScratchFloats) + " floats";
    return SPX_ERR_ARG;
  }
  float* scratch = nullptr;
  if (int rc = scratch_for_current_device(&scratch)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  spx::Grid g{(int)size_x, (int)size_y, (int)size_x + 2, 0, 0};
  if (n_pass == 0) {
    if (d_out != d_in && cudaMemcpyAsync(d_out, d_in, cells * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
      g_noalloc_err = "spx_filter_noalloc: device copy failed";
      return SPX_ERR_CUDA;
    }
    return SPX_OK;
  }
  // Passes alternate between d_out and the scratch so that the last one lands
  // in d_out.  An in-place call (d_in == d_out) starts in the scratch and, for
  // an odd pass count, copies the result back at the end.
  const float* src = d_in;
  float* dst;
  const bool in_place = d_in == d_out;
  bool to_out = in_place ? false : (n_pass % 2 == 1);
  for (uint32_t p = 0; p < n_pass; ++p) {
    dst = to_out ? d_out : scratch;
    float* s = const_cast<float*>(src);
    spx::launch_filter_pass(g, &s, &dst, 1, st);
    src = dst;
    to_out = !to_out;
  }
  if (src != d_out &&
      cudaMemcpyAsync(d_out, src, cells * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
    g_noalloc_err = "spx_filter_noalloc: device copy failed";
    return SPX_ERR_CUDA;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_noalloc_err = std::string("spx_filter_noalloc: launch failed: ") + cudaGetErrorString(e);
    return SPX_ERR_CUDA;
  }
  return SPX_OK;
}
