// Membrane Hessian-vector product for callers that cannot allocate device memory.
//
// Some hosts may not call cudaMalloc while they step the cloth: a caller that
// records its frame into a CUDA graph (allocation is not allowed during stream
// capture), a real-time render loop that cannot afford the device-wide
// synchronization cudaMalloc implies, or a plugin whose device memory belongs to
// another runtime's pool. This entry point lets them compute the same product as
// cs_membrane_hvp without creating a solver handle: they pass device pointers for
// every input and for the output, and the scratch the kernels need lives in one
// fixed-size array in the library's own device image.
//
// The array is a file-scope __device__ object, so every GPU that loads this
// library holds it (about 11 MB) until the process exits. All calls share it and
// it keeps the contents of the last call; calls that overlap on the GPU (two
// streams, or two host threads) race on it and must be serialized by the caller.
// Nothing in it needs to start at zero: each call writes every scratch word it
// reads before reading it.
#include <mutex>

#include "../../include/closim_cuda.h"
#include "plain.cuh"

namespace cs {

constexpr size_t kStaticElem = 18ull * CS_STATIC_HVP_MAX_TRIANGLES;  // per-triangle FD gradients
constexpr size_t kStaticTerms = 3ull * CS_STATIC_HVP_MAX_VERTICES;   // |p|^2 terms
constexpr size_t kStaticDoubles = kStaticElem + kStaticTerms + 32;   // + the step size h

static __device__ __align__(256) double g_hvp_scratch[kStaticDoubles];

namespace {
std::mutex g_setup_mu;
double* g_scratch_ptr[64] = {};  // device address of g_hvp_scratch, per device
}  // namespace

// Resolves the array's device address on the current device (once per device).
// The address is cached by device index for the life of the process; a
// cudaDeviceReset unloads the library's device image and leaves the cache
// stale, so the entry point is not for processes that reset a device.
static int scratch_on_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CS_E_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_hvp_scratch) != cudaSuccess || !p) return CS_E_CUDA;
    g_scratch_ptr[dev] = (double*)p;
  }
  *out = g_scratch_ptr[dev];
  return CS_OK;
}

}  // namespace cs

extern "C" int cs_membrane_hvp_static(int32_t n, int32_t m, const uint32_t* indices, const float* inv_dm,
                                      const float* area, const uint32_t* inc_offsets, const uint32_t* inc_records,
                                      const cs_material* mat, const double* x, const double* p, double* out,
                                      void* stream) {
  if (n <= 0 || m <= 0 || !indices || !inv_dm || !area || !inc_offsets || !inc_records || !mat || !x || !p || !out)
    return CS_E_ARG;
  if ((reinterpret_cast<uintptr_t>(inv_dm) & 15u) != 0) return CS_E_ARG;  // read as float4 per triangle
  if (n > CS_STATIC_HVP_MAX_VERTICES || m > CS_STATIC_HVP_MAX_TRIANGLES) return CS_E_CAPACITY;
  double* scratch = nullptr;
  const int rc = cs::scratch_on_current_device(&scratch);
  if (rc != CS_OK) return rc;
  double* elem = scratch;
  double* terms = scratch + cs::kStaticElem;
  double* h = terms + cs::kStaticTerms;
  const cs::Mat<double> mt{mat->stretch_warp, mat->stretch_weft, mat->stretch_coupling, mat->shear, mat->thickness};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cs::launch_membrane_hvp(indices, reinterpret_cast<const float4*>(inv_dm), area, mt, n, m, inc_offsets, inc_records,
                          x, p, out, terms, h, elem, s);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}
