// gr_host.h -- internal host-side declarations shared by the C-ABI translation units.
#pragma once

#include <cstddef>
#include <cstdint>

#include "gemray_cuda.h"

namespace grh {

// A lazily grown device allocation owned by a context (the reference's
// `ensure_capacity`, renderer/gpu/frame.rs:868-879).
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t cap = 0;
    gr_status reserve(size_t bytes);
    void release();
};

// Device tone map (gr_tonemap.cu): rgba_dev[i] = sRGB ACES encode of xyz_dev[i] * scale.
gr_status tonemap_device(const float *xyz_dev, float scale, uint32_t n, void *rgba_dev, struct CUstream_st *s);

// evaluate_gem_optical_metrics for a batch of poses on `s` (gr_metrics.cu); host
// `out` is written before it returns.  Requires n_planes > 0.
gr_status metrics_device(const gr_plane *planes, uint32_t n_planes, const gr_material *m, const gr_pose *poses,
                         uint32_t n_poses, gr_metrics_out *out, uint32_t flags, struct CUstream_st *s,
                         DeviceBuffer &scratch);
// Device scratch bytes metrics_device needs (a scratch at least this large never grows).
size_t metrics_scratch_bytes(uint32_t n_planes, uint32_t n_poses);

// The fixed scratch of gr_render_resident_static (gr_static.cu): its address on
// `device` (the current device), looked up once per device.  Returns a cudaError_t.
constexpr int kStaticMaxDevices = 64;
int static_scratch(int device, float **out);

}  // namespace grh
