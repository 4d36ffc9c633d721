// gr_static.cu -- the fixed device scratch behind gr_render_resident_static.
//
// One file-scope device array holds the per-tuple XYZ (3 f32 per tuple) of one pixel
// chunk.  The module loader places it once per device, so a render that uses it
// allocates no device memory at call time.  The array lives in its own translation
// unit (no kernels here): under lazy module loading its 16 MiB are only placed on a
// device when the address is first looked up.
#include <cuda_runtime.h>

#include <mutex>

#include "gemray_cuda.h"
#include "gr_host.h"

static __device__ __align__(256) float g_static_xyz[GR_STATIC_SCRATCH_BYTES / sizeof(float)];

static_assert((size_t)GR_STATIC_SCRATCH_TUPLES * 3 * sizeof(float) <= GR_STATIC_SCRATCH_BYTES,
              "the scratch holds GR_STATIC_SCRATCH_TUPLES tuples");

namespace {
std::mutex g_mu;
float *g_addr[grh::kStaticMaxDevices];
}  // namespace

namespace grh {

int static_scratch(int device, float **out) {
    *out = nullptr;
    if (device < 0 || device >= kStaticMaxDevices) return (int)cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_xyz);
        if (e != cudaSuccess) return (int)e;
        g_addr[device] = (float *)p;
    }
    *out = g_addr[device];
    return (int)cudaSuccess;
}

}  // namespace grh
