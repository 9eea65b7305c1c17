// Allocation-free relaxation of one small gridshell.
//
// Some callers cannot allocate device memory on their own: a host whose framework owns every byte of the GPU through
// its own pool or caching allocator (a cudaMalloc behind its back fragments that pool or breaks its budget), a process
// that must not allocate once it is serving (allocation can stall or fail at run time), or an application that has
// measured and frozen its memory up front.  ws_relax_noalloc serves them: the whole device footprint of one instance
// (its arena, descriptor and control block) lives in the file-scope array below, which every GPU that loads this
// library holds, WS_NOALLOC_SCRATCH_BYTES of it, until the process exits.  The call allocates no device memory.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/weavesim.h"
#include "errors.hpp"
#include "host_goals.hpp"

namespace wsb {
size_t instanceFootprint(int prec, const HostGoals &g);
int runInPlace(int prec, const HostGoals &g, char *base, int nIter, int threads, cudaStream_t st, ws_state_out *out,
               ws_control *ctl, std::string &err);
}  // namespace wsb

static __device__ __align__(256) unsigned char g_noalloc_scratch[WS_NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_mu;                          // host calls take turns: every call uses the same array

// the array's device address on the current device: in host code the symbol is only a host-side stand-in, so the
// address comes from cudaGetSymbolAddress.  It is looked up on every call (cheap once the device code is loaded), so
// a device reset that reloads the module at another address cannot leave a stale pointer behind.
int scratchAddress(void **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return wsb::fail(WS_ERR_CUDA, std::string("ws_relax_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
  *out = p;
  return WS_OK;
}
}  // namespace

extern "C" int ws_relax_noalloc(const ws_model *model, int32_t precision, int32_t n_iter, int32_t threads, void *stream,
                                ws_state_out *out, ws_control *ctl) {
  if (!model || n_iter < 0) return wsb::fail(WS_ERR_ARG, "ws_relax_noalloc: null model or negative iteration count");
  if (precision < 0 || precision > 2) return wsb::fail(WS_ERR_ARG, "ws_relax_noalloc: unknown precision");
  if (threads == 0) threads = 256;
  if (threads < 32 || threads > 512 || (threads % 32)) return wsb::fail(WS_ERR_ARG, "ws_relax_noalloc: threads must be a multiple of 32 up to 512");
  wsb::HostGoals g;
  try {
    g.build(*model);
  } catch (const std::exception &e) {
    return wsb::fail(WS_ERR_ARG, std::string("ws_relax_noalloc: ") + e.what());
  }
  const size_t need = wsb::instanceFootprint(precision, g);
  if (need > WS_NOALLOC_SCRATCH_BYTES)
    return wsb::fail(WS_ERR_ARG, "ws_relax_noalloc: the model needs " + std::to_string(need) + " bytes of device scratch; this "
                     "entry point holds " + std::to_string(size_t(WS_NOALLOC_SCRATCH_BYTES)) + " (use ws_create for larger models)");
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return wsb::fail(WS_ERR_NODEV, std::string("ws_relax_noalloc: no CUDA device: ") + cudaGetErrorString(e));
  if (stream) {
    // the scratch address belongs to the current device: a stream of another device would run on the wrong memory
    int sdev = -1;
    e = cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &sdev);
    if (e != cudaSuccess) return wsb::fail(WS_ERR_ARG, std::string("ws_relax_noalloc: bad stream: ") + cudaGetErrorString(e));
    if (sdev != dev)
      return wsb::fail(WS_ERR_ARG, "ws_relax_noalloc: the stream belongs to device " + std::to_string(sdev) +
                       ", the current device is " + std::to_string(dev));
  }
  void *base = nullptr;
  int rc = scratchAddress(&base);
  if (rc != WS_OK) return rc;
  std::string err;
  rc = wsb::runInPlace(precision, g, static_cast<char *>(base), n_iter, threads, static_cast<cudaStream_t>(stream), out, ctl, err);
  if (rc != WS_OK) return wsb::fail(rc, "ws_relax_noalloc: " + err);
  return WS_OK;
}
