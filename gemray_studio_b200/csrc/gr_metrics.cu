// gr_metrics.cu -- brilliance / fire / scintillation / windowing / extinction out,
// = evaluate_gem_optical_metrics (crates/gemray/src/color/metrics.rs:1082-1237) for
// a batch of poses (tilt sweeps, metrics.rs:1262-1289, are batches of poses).
//
// k_metric_samples: one thread per (pose, grid cell, slot); slots 0..4 are the five
//   aperture rays of classify_aperture_sample (metrics.rs:568-676: a d-line trace,
//   then F- and C-line traces for returned rays), slots 5..9 the five yaw offsets of
//   cell_temporal_variance (metrics.rs:349-380).  Results land in a per-sample array.
// k_metric_reduce: one thread per pose folds the samples in the reference's order
//   (cells ix-major, then aperture order) with the reference's f32 arithmetic, so the
//   counts are exact and the f32 sums are formed in the same sequence.
// Camera bases, the studio rig and the d/F/C indices are host-computed per pose with
// the reference's f32 libm arithmetic.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "gemray_cuda.h"
#include "gr_host.h"
#include "gr_trace.cuh"

namespace grd {

constexpr int MGRID = 18;
constexpr int MSLOTS = 10;

struct PoseConst {
    float fwd[3], right[3], up[3];         // camera_view_basis(cam_yaw, cam_pitch)
    float tf[5][3], tr[5][3], tu[5][3];    // bases at the five temporal yaw offsets
    float key[3], fill[3], sin_lp;         // StudioRig::new(light_yaw, light_pitch)
    float nd, nf, nc;                      // indices at 589.3 / 486.1 / 656.3 nm
};

struct MetricSample {
    uint32_t cls;   // 0 no hit, 1 entry blocked, 2 windowed, 3 extinct, 4 returned; temporal: 0/1
    uint32_t fire_valid;
    float angle_deg, weight;
};

// metrics.rs:118-131
__device__ __forceinline__ float m_fresnel_t(float n1, float n2, float ci, float ct) {
    float ds = fmaf(n2, ct, n1 * ci), dp = fmaf(n2, ci, n1 * ct);
    if (fabsf(ds) < 1e-6f || fabsf(dp) < 1e-6f) return 0.0f;
    float a = fmaf(n2, -ct, n1 * ci) / ds, b = fmaf(n2, -ci, n1 * ct) / dp;
    return clampf(1.0f - midpoint(a * a, b * b), 0.0f, 1.0f);
}

struct MExit {
    V3 dir;
    float transmittance, exit_cos;
    int facet;
    uint32_t bounces;
};

// metrics.rs:138-227 (fates: 0 blocked, 1 leaked, 2 exited upward, 3 absorbed)
__device__ int m_trace_wavelength(V3 entry, V3 in_dir, V3 n_entry, float cos_i, const float4 *planes, uint32_t n,
                                  float index, MExit &ex) {
    float sin2_t = (1.0f / (index * index)) * fmaf(cos_i, -cos_i, 1.0f);
    if (sin2_t > 1.0f) return 0;
    float cos_t = sqrtf(1.0f - sin2_t);
    V3 dir = normalize(add(smul(1.0f / index, in_dir), smul(fmaf(1.0f / index, cos_i, -cos_t), n_entry)));
    V3 hp = add(entry, mul(dir, 1e-4f));
    float sin_crit = 1.0f / index;
    float entry_t = m_fresnel_t(1.0f, index, cos_i, cos_t);
    bool leaked = false, up = false;
    for (uint32_t bounce = 0; bounce < 10; ++bounce) {
        float t = 0.0f;
        int idx = 0;
        if (!intersect(planes, n, hp, dir, t, idx)) break;
        V3 np = add(hp, smul(t, dir));
        V3 n_out = plane_normal(planes, idx);
        float ct = clampf(dot(dir, n_out), 0.0f, 1.0f);
        float st = sqrtf(fmaxf(fmaf(ct, -ct, 1.0f), 0.0f));
        if (st < sin_crit) {
            float s2o = (index * index) * fmaf(ct, -ct, 1.0f);
            if (s2o <= 1.0f) {
                float co = sqrtf(1.0f - s2o);
                V3 od = normalize(add(smul(index, dir), smul(fmaf(index, -ct, co), n_out)));
                if (n_out.y < -0.05f) {
                    leaked = true;
                } else if (od.y > 0.05f) {
                    up = true;
                    ex.dir = od;
                    ex.transmittance = m_fresnel_t(index, 1.0f, ct, co);
                    ex.exit_cos = co;
                    ex.facet = idx < 0 ? 0 : idx;
                    ex.bounces = bounce;
                }
                break;
            }
        }
        dir = normalize(sub(dir, smul(2.0f * ct, n_out)));
        hp = add(np, mul(dir, 1e-4f));
    }
    if (leaked) return 1;
    if (up) {
        ex.transmittance = entry_t * ex.transmittance;
        return 2;
    }
    return 3;
}

// metrics.rs:229-252
__device__ __forceinline__ bool m_visible(V3 d, V3 fwd, const PoseConst &P) {
    bool head = dot(neg(d), fwd) > 0.96f;
    float kd = fmaxf(dot(d, ld3(P.key)), 0.0f), fd = fmaxf(dot(d, ld3(P.fill)), 0.0f);
    bool ring = fabsf(fmaf(P.sin_lp, -0.8f, d.y)) < 0.35f;
    bool lit = (kd > 0.70f) || (fd > 0.75f) || (ring && d.y > 0.2f);
    return !head && lit;
}

__device__ __forceinline__ bool cell_uv(int ix, int iz, float &u, float &v) {
    u = fmaf(((float)ix + 0.5f) / (float)MGRID, 2.0f, -1.0f);
    v = fmaf(((float)iz + 0.5f) / (float)MGRID, 2.0f, -1.0f);
    return !(fmaf(v, v, u * u) > 0.70f);
}

__global__ void k_metric_samples(const PoseConst *__restrict__ poses, uint32_t n_poses, const float4 *__restrict__ gplanes,
                                 uint32_t n_planes, MetricSample *__restrict__ out) {
    extern __shared__ float4 s_planes[];
    for (uint32_t i = threadIdx.x; i < n_planes; i += blockDim.x) s_planes[i] = gplanes[i];
    __syncthreads();
    const uint32_t per_pose = MGRID * MGRID * MSLOTS;
    const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (uint64_t)n_poses * per_pose) return;
    const uint32_t pose = (uint32_t)(gid / per_pose);
    const uint32_t rem = (uint32_t)(gid % per_pose);
    const uint32_t cell = rem / MSLOTS, slot = rem % MSLOTS;
    const int ix = (int)(cell / MGRID), iz = (int)(cell % MGRID);
    MetricSample r{0u, 0u, 0.0f, 0.0f};
    float u, v;
    if (!cell_uv(ix, iz, u, v)) {
        out[gid] = r;
        return;
    }
    const PoseConst &P = poses[pose];
    if (slot < 5) {
        // classify_aperture_sample (metrics.rs:568-676)
        const float ap[5][2] = {{0.f, 0.f}, {0.08f, 0.f}, {-0.08f, 0.f}, {0.f, 0.08f}, {0.f, -0.08f}};
        V3 fwd = ld3(P.fwd), right = ld3(P.right), upv = ld3(P.up);
        V3 rd = normalize(add(add(fwd, smul(ap[slot][0], right)), smul(ap[slot][1], upv)));
        V3 ro = add(add(mul(neg(fwd), 2.5f), smul(u * 0.95f, right)), smul(v * 0.95f, upv));
        float t = 0.0f;
        int idx = 0;
        if (intersect(s_planes, n_planes, ro, rd, t, idx)) {
            V3 hp = add(ro, smul(t, rd));
            V3 nrm = plane_normal(s_planes, idx);
            float ci = clampf(dot(neg(rd), nrm), 0.0f, 1.0f);
            MExit e;
            int fate = m_trace_wavelength(hp, rd, nrm, ci, s_planes, n_planes, P.nd, e);
            if (fate == 0) r.cls = 1;
            else if (fate == 1) r.cls = 2;
            else if (fate == 3) r.cls = 3;
            else if (!m_visible(e.dir, fwd, P)) r.cls = 3;
            else {
                r.cls = 4;
                MExit ef, ec;
                int ff = m_trace_wavelength(hp, rd, nrm, ci, s_planes, n_planes, P.nf, ef);
                int fc = m_trace_wavelength(hp, rd, nrm, ci, s_planes, n_planes, P.nc, ec);
                if (ff == 2 && fc == 2 && ef.facet == ec.facet && ef.bounces == ec.bounces) {
                    float cs = clampf(dot(ef.dir, ec.dir), -1.0f, 1.0f);
                    r.angle_deg = m_acos(cs) * 57.2957795130823208767981548141051703f;
                    r.weight = (e.transmittance * ef.transmittance * ec.transmittance) *
                               (fmaxf(ef.exit_cos, 0.0f) * fmaxf(ec.exit_cos, 0.0f));
                    r.fire_valid = 1;
                }
            }
        }
    } else {
        // cell_returned_at_yaw_offset (metrics.rs:295-330)
        const uint32_t k = slot - 5;
        V3 f2 = ld3(P.tf[k]), r2 = ld3(P.tr[k]), u2 = ld3(P.tu[k]);
        V3 ro = add(add(mul(neg(f2), 2.5f), smul(u * 0.95f, r2)), smul(v * 0.95f, u2));
        float t = 0.0f;
        int idx = 0;
        if (intersect(s_planes, n_planes, ro, f2, t, idx)) {
            V3 hp = add(ro, smul(t, f2));
            V3 nrm = plane_normal(s_planes, idx);
            float ci = clampf(dot(neg(f2), nrm), 0.0f, 1.0f);
            MExit e;
            if (m_trace_wavelength(hp, f2, nrm, ci, s_planes, n_planes, P.nd, e) == 2 && m_visible(e.dir, f2, P))
                r.cls = 1;
        }
    }
    out[gid] = r;
}

// The reference's accumulation order (metrics.rs:1127-1236) per pose.
__global__ void k_metric_reduce(const MetricSample *__restrict__ in, uint32_t n_poses, gr_metrics_out *__restrict__ out,
                                uint32_t use_fp64) {
    const uint32_t pose = blockIdx.x * blockDim.x + threadIdx.x;
    if (pose >= n_poses) return;
    const MetricSample *s = in + (size_t)pose * MGRID * MGRID * MSLOTS;
    uint32_t total = 0, windowed = 0, extinct = 0, returned = 0, cell_count = 0;
    float fire_sum = 0.f, cf_sum = 0.f, cf_sq = 0.f, tv_sum = 0.f;
    double fire_d = 0.0, cf_d = 0.0, cf_sq_d = 0.0, tv_d = 0.0;
    for (int ix = 0; ix < MGRID; ++ix) {
        for (int iz = 0; iz < MGRID; ++iz) {
            float u, v;
            if (!cell_uv(ix, iz, u, v)) continue;
            const MetricSample *c = s + (size_t)(ix * MGRID + iz) * MSLOTS;
            uint32_t ct_total = 0, ct_ret = 0;
            for (int a = 0; a < 5; ++a) {
                const MetricSample &m = c[a];
                if (m.cls == 0) continue;
                total++;
                ct_total++;
                if (m.cls == 2) windowed++;
                else if (m.cls == 3) extinct++;
                else if (m.cls == 4) {
                    returned++;
                    ct_ret++;
                    if (m.fire_valid) {
                        fire_sum = fmaf(m.angle_deg, m.weight, fire_sum);
                        fire_d = fma((double)m.angle_deg, (double)m.weight, fire_d);
                    }
                }
            }
            if (ct_total > 0) {
                float frac = (float)ct_ret / (float)ct_total;
                cf_sum += frac;
                cf_sq = fmaf(frac, frac, cf_sq);
                cf_d += (double)frac;
                cf_sq_d = fma((double)frac, (double)frac, cf_sq_d);
                cell_count++;
                uint32_t tr = 0;
                for (int k = 0; k < 5; ++k) tr += c[5 + k].cls;
                float tp = (float)tr / 5.0f;
                tv_sum += fmaf(tp, -tp, tp);
                tv_d += (double)fmaf(tp, -tp, tp);
            }
        }
    }
    if (use_fp64) {
        fire_sum = (float)fire_d;
        cf_sum = (float)cf_d;
        cf_sq = (float)cf_sq_d;
        tv_sum = (float)tv_d;
    }
    const float nt = (float)(total > 1 ? total : 1);
    gr_metrics_out o;
    o.windowing_pct = clampf((float)windowed / nt * 100.0f, 0.0f, 100.0f);
    o.extinction_pct = clampf((float)extinct / nt * 100.0f, 0.0f, 100.0f);
    o.brilliance_pct = clampf((float)returned / nt * 100.0f, 0.0f, 100.0f);
    o.fire_index = fmaxf(fire_sum / nt * 275.0f, 0.1f);
    float spatial = 0.0f;
    if (cell_count > 0) {
        float mean = cf_sum / (float)cell_count;
        if (mean > 1e-4f) {
            float var = fmaxf(fmaf(mean, -mean, cf_sq / (float)cell_count), 0.0f);
            float cv = sqrtf(var) / mean;
            spatial = clampf(cv / (1.0f + cv) * 100.0f, 0.0f, 100.0f);
        }
    }
    float temporal = cell_count > 0 ? clampf((tv_sum / (float)cell_count) / 0.24f * 100.0f, 0.0f, 100.0f) : 0.0f;
    o.scintillation_pct = clampf(fmaf(0.4f, temporal, 0.6f * spatial), 0.0f, 100.0f);
    out[pose] = o;
}

}  // namespace grd

namespace {

struct H3 {
    float x, y, z;
};
inline float hdot(H3 a, H3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline H3 hnorm(H3 a) {
    float r = 1.0f / sqrtf(hdot(a, a));
    return H3{a.x * r, a.y * r, a.z * r};
}
inline H3 hcross(H3 a, H3 b) { return H3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }

// metrics.rs:16-30
void camera_view_basis(float yaw, float pitch, float f[3], float r[3], float u[3]) {
    float cp = cosf(pitch), sp = sinf(pitch), cy = cosf(yaw), sy = sinf(yaw);
    H3 fw = hnorm(H3{-cp * sy, -sp, -cp * cy});
    H3 wu = fabsf(cp) < 1e-4f ? H3{0.f, 0.f, -1.f} : H3{0.f, 1.f, 0.f};
    H3 rt = hnorm(hcross(fw, wu));
    H3 up = hnorm(hcross(rt, fw));
    f[0] = fw.x; f[1] = fw.y; f[2] = fw.z;
    r[0] = rt.x; r[1] = rt.y; r[2] = rt.z;
    u[0] = up.x; u[1] = up.y; u[2] = up.z;
}

float host_dispersion(const gr_dispersion &d, float lambda_nm) {  // optics/dispersion.rs:12-37
    float lum = lambda_nm * 1e-3f, l2 = lum * lum;
    if (d.model_type == GR_DISP_SELLMEIER1) return sqrtf(fmaxf(1.0f + (d.param_a[0] * l2) / (l2 - d.param_b[0]), 1.0f));
    if (d.model_type == GR_DISP_SELLMEIER3) {
        float n2 = 1.0f;
        n2 = n2 + (d.param_a[0] * l2) / (l2 - d.param_b[0]);
        n2 = n2 + (d.param_a[1] * l2) / (l2 - d.param_b[1]);
        n2 = n2 + (d.param_a[2] * l2) / (l2 - d.param_b[2]);
        return sqrtf(fmaxf(n2, 1.0f));
    }
    float l4 = l2 * l2;
    return d.param_a[0] + (d.param_a[1] / l2) + (d.param_a[2] / l4);
}

}  // namespace

namespace grh {
void studio_rig(float yaw, float pitch, float key[3], float fill[3], float ring[16][3]);

namespace {
struct MetricsLayout {
    size_t pose_bytes, plane_bytes, sample_bytes, out_bytes;
    size_t total() const { return pose_bytes + plane_bytes + sample_bytes + out_bytes; }
};
MetricsLayout metrics_layout(uint32_t n_planes, uint32_t n_poses) {
    const size_t per_pose = (size_t)grd::MGRID * grd::MGRID * grd::MSLOTS;
    MetricsLayout L;
    L.pose_bytes = ((n_poses * sizeof(grd::PoseConst)) + 255) & ~(size_t)255;
    L.plane_bytes = (((size_t)(n_planes ? n_planes : 1) * sizeof(float4)) + 255) & ~(size_t)255;
    L.sample_bytes = ((n_poses * per_pose * sizeof(grd::MetricSample)) + 255) & ~(size_t)255;
    L.out_bytes = n_poses * sizeof(gr_metrics_out);
    return L;
}
}  // namespace

size_t metrics_scratch_bytes(uint32_t n_planes, uint32_t n_poses) { return metrics_layout(n_planes, n_poses).total(); }

gr_status metrics_device(const gr_plane *planes, uint32_t n_planes, const gr_material *m, const gr_pose *poses,
                         uint32_t n_poses, gr_metrics_out *out, uint32_t flags, cudaStream_t stream, DeviceBuffer &scratch) {
    std::vector<grd::PoseConst> pc(n_poses);
    const float nd = fmaxf(host_dispersion(m->dispersion, 589.3f), 1.1f);
    const float nf = fmaxf(host_dispersion(m->dispersion, 486.1f), 1.001f);
    const float nc = fmaxf(host_dispersion(m->dispersion, 656.3f), 1.001f);
    const float yaw_off[5] = {-3.0f, -1.5f, 0.0f, 1.5f, 3.0f};
    const float deg2rad = 3.14159265358979323846f / 180.0f;
    for (uint32_t i = 0; i < n_poses; ++i) {
        grd::PoseConst &P = pc[i];
        camera_view_basis(poses[i].cam_yaw, poses[i].cam_pitch, P.fwd, P.right, P.up);
        for (int k = 0; k < 5; ++k)
            camera_view_basis(poses[i].cam_yaw + yaw_off[k] * deg2rad, poses[i].cam_pitch, P.tf[k], P.tr[k], P.tu[k]);
        float ring[16][3];
        studio_rig(poses[i].light_yaw, poses[i].light_pitch, P.key, P.fill, ring);
        P.sin_lp = sinf(poses[i].light_pitch);
        P.nd = nd;
        P.nf = nf;
        P.nc = nc;
    }
    const size_t per_pose = (size_t)grd::MGRID * grd::MGRID * grd::MSLOTS;
    const MetricsLayout L = metrics_layout(n_planes, n_poses);
    const size_t pose_bytes = L.pose_bytes, plane_bytes = L.plane_bytes, sample_bytes = L.sample_bytes,
                 out_bytes = L.out_bytes;
    gr_status st = scratch.reserve(L.total());
    if (st != GR_OK) return st;
    char *base = (char *)scratch.ptr;
    grd::PoseConst *d_pose = (grd::PoseConst *)base;
    float4 *d_planes = (float4 *)(base + pose_bytes);
    grd::MetricSample *d_samp = (grd::MetricSample *)(base + pose_bytes + plane_bytes);
    gr_metrics_out *d_out = (gr_metrics_out *)(base + pose_bytes + plane_bytes + sample_bytes);
    if (cudaMemcpyAsync(d_pose, pc.data(), n_poses * sizeof(grd::PoseConst), cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return GR_ECUDA;
    if (n_planes && cudaMemcpyAsync(d_planes, planes, n_planes * sizeof(gr_plane), cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return GR_ECUDA;
    const uint64_t threads = (uint64_t)n_poses * per_pose;
    const unsigned T = 128;
    grd::k_metric_samples<<<(unsigned)((threads + T - 1) / T), T, n_planes * sizeof(float4), stream>>>(
        d_pose, n_poses, d_planes, n_planes, d_samp);
    grd::k_metric_reduce<<<(n_poses + 63) / 64, 64, 0, stream>>>(d_samp, n_poses, d_out,
                                                                 (flags & GR_METRICS_FP64_SUMS) ? 1u : 0u);
    if (cudaGetLastError() != cudaSuccess) return GR_ECUDA;
    if (cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, stream) != cudaSuccess) return GR_ECUDA;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return GR_ECUDA;
    return GR_OK;
}
}  // namespace grh
