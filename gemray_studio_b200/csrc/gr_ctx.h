// gr_ctx.h -- the engine context and resident scenes, shared by the host translation
// units (gr_host.cu, gr_batch.cu).  Internal: not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "gemray_cuda.h"
#include "gr_device.cuh"
#include "gr_host.h"

using grd::SceneConst;

namespace grh {
// Records a formatted message for gr_last_error_string() and returns st.
gr_status fail(gr_status st, const char *fmt, ...);
}  // namespace grh

#define GR_CUDA(call)                                                                                       \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return grh::fail(GR_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Bounce caps of the staged kernels' first two stages ({0, 0} = the built-in pair) and
// the resident blocks per SM their register allocation targets (0 = the built-in
// GR_TRACE_MIN_BLOCKS): a staged schedule.
struct StageCaps {
    uint32_t first = 0, second = 0;
    uint32_t blocks = 0;
};
// Blocks-per-SM targets the staged single-scene kernels are built for: [0] is the
// built-in one.  Measured on B200 (c2 / c3 frames): 10 blocks (48 registers) 2.3%
// faster than 9 (56) on both, 7 and 8 slower.
constexpr uint32_t kScheduleBlocks[2] = {GR_TRACE_MIN_BLOCKS, 10};

// The staged schedule (stage caps and blocks per SM) a stone's staged renders use.
// Every schedule gives the same films, but the fastest depends on the stone's path
// lengths and register pressure, so from the stone's second staged call on, one call
// with each candidate schedule is timed on the device (the whole call: its chunks cover
// different parts of the image) and the schedule with the least time per tuple is kept
// (gr_host.cu, kScheduleCandidates).
struct StageCapTune {
    static constexpr int kCandidates = 6;
    int best = -1;              // chosen candidate, -1 while measuring
    uint32_t staged_calls = 0;  // staged calls seen
    bool issued[kCandidates] = {};
    float ms_per_mtuple[kCandidates] = {3.0e38f, 3.0e38f, 3.0e38f, 3.0e38f, 3.0e38f,
                                        3.0e38f};  // unmeasured: never chosen over a measured one
    struct Trial {
        cudaEvent_t start = nullptr, stop = nullptr;
        int candidate = 0;
        uint64_t tuples = 0;
        bool done = false;
    } trial[kCandidates];
};

struct ResidentScene {
    SceneConst S;
    grh::DeviceBuffer planes, map, ext;
    uint64_t bytes = 0;
    uint32_t users = 0;  // open frame streams rendering this scene (gr_stream.cu)
    StageCapTune tune;
};

struct FrameStream;  // gr_stream.cu

struct ServeState;  // gr_serve.cu

// A captured batch launch sequence and the batch shape it is valid for.
struct BatchGraph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec;
};
constexpr size_t kMaxBatchGraphs = 16;

struct gr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    std::string label;
    size_t chunk_budget = 2048ull << 20;
    uint64_t serve_budget = 60ull << 30;
    int sm_count = 0;
    grh::DeviceBuffer xyz, film, planes, map, ext, counter, rgba, metrics;
    int kernel_mode = GR_KERNEL_AUTO;
    // staged kernels' park buffer (count word, then parked path records)
    grh::DeviceBuffer park;
    // Optional per-launch timing of the trace and fold kernels (CUDA events on the
    // launch stream); read back by gr_timing_read.
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> trace_ev, fold_ev;
    // gr_accumulate's stage-cap choices, keyed by the stone (planes, finishes, material,
    // depth, flags: what sets the path lengths); cleared past kMaxAccumTunes stones
    std::map<uint64_t, StageCapTune> accum_tune;
    static constexpr size_t kMaxAccumTunes = 64;
    size_t trace_used = 0, fold_used = 0;
    uint64_t trace_launches = 0, fold_launches = 0;
    // gr_render_batch: scene-slot + segment tables, captured launch sequences, and a
    // ring of pinned host staging buffers for the table uploads (a pageable source
    // would make each upload wait for the previous batch to reach its copy)
    grh::DeviceBuffer batch_tables, batch_park;  // segment tables; staged park records + slot counters
    static constexpr int kStageSlots = 4;
    void *stage_host[kStageSlots] = {};
    size_t stage_cap[kStageSlots] = {};
    cudaEvent_t stage_ev[kStageSlots] = {};
    int stage_next = 0;
    std::vector<BatchGraph> batch_graphs;
    // gr_submit / gr_poll request loop (created by the first submit)
    ServeState *serve = nullptr;
    std::map<uint64_t, ResidentScene *> scenes;
    uint64_t next_scene_id = 1;
    // gr_stream_* frame-delta streams (gr_stream.cu)
    std::map<uint64_t, FrameStream *> streams;
    uint64_t next_stream_id = 1;
    // guide pass and A-Trous scratch (gr_denoise.cu)
    grh::DeviceBuffer dn_a, dn_b, dn_n, dn_g, dn_in, dn_out, dn_planes;
    cudaEvent_t dn_ev = nullptr;
    uint64_t resident_bytes = 0;
};

// Device pointers of a resident scene in the layout the kernels take.
grd::SceneBuffers resident_buffers(ResidentScene *rs);

namespace grh {
// One batch item plus its fold mode: cont = 0 adds each call's per-pixel sum once
// (gr_render_batch); cont = 1 continues the film's running sum (serving slices; comp
// holds the Kahan compensation for scenes with GR_FLAG_KAHAN_FILM).
struct BatchItem {
    gr_batch_item it;
    float *comp;
    uint32_t cont;
};
// gr_render_batch's body; the caller holds ctx->mu and has made ctx->device current.
gr_status batch_enqueue(gr_ctx *ctx, const BatchItem *items, uint32_t n_items, uint32_t flags, cudaStream_t stream);
}  // namespace grh

namespace grh {
// Stops the request loop and frees its requests; the caller holds no lock.
void serve_shutdown(gr_ctx *ctx);
// Cancels, joins and frees every frame stream; the caller holds no lock.
void streams_shutdown(gr_ctx *ctx);
}  // namespace grh

namespace grd {
struct LaunchRange;
struct Path;
}
namespace grh {
// Scene checks and encoding (gr_host.cu): validate, encode the constants, and upload
// the scene's arrays into the context's buffers (prepare does all three).
gr_status validate_scene(const gr_scene *sc);
void encode_scene(const gr_scene *sc, SceneConst &S);
gr_status prepare(gr_ctx *ctx, const gr_scene *sc, SceneConst &S, grd::SceneBuffers &B);
// Tuples [0, R.n_tuples) of one chunk traced into xyz on `stream` with kernel `mode`
// (gr_host.cu), and the ordered per-pixel fold of n_pixels pixels into film.
// STAGED mode parks paths in `park` (the context's buffer when NULL).
gr_status launch_trace(gr_ctx *ctx, const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R,
                       float *xyz, cudaStream_t stream, int mode, grh::DeviceBuffer *park = nullptr,
                       StageCaps caps = StageCaps{});
// The compile-time scene class of a single-scene launch (gr_trace.cuh K_*): clear
// isotropic stones (K_ISO | K_CLEAR) and the rest, each with its environment kind;
// -1 for scenes the extension variant handles (frosted, scattering, biaxial).
int scene_class(const SceneConst &S);
// Park buffers and caps of a staged single-scene launch (prepared by launch_trace).
struct StagedLaunch {
    grd::Path *park1, *park2;
    unsigned int *counts;
    uint64_t cap1, cap2;
    uint32_t cap_first, cap_second;
    uint32_t blocks;  // kScheduleBlocks entry, 0 = the built-in one
};
// The plain kernel (st == NULL) or the three staged launches of scene class K
// (gr_single_clear.cu / gr_single_general.cu).
// sorted_work != NULL: the block-sorted kernel (gr_sorted.cuh) instead, its tuple counter.
gr_status launch_single_clear(int K, const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R,
                              float *xyz, cudaStream_t stream, const StagedLaunch *st,
                              unsigned int *sorted_work = nullptr, int sm_count = 0);
gr_status launch_single_general(int K, const SceneConst &S, const grd::SceneBuffers &B, const grd::LaunchRange &R,
                                float *xyz, cudaStream_t stream, const StagedLaunch *st);
// The kernel a launch of n_tuples tuples runs in `mode` (AUTO resolved by size), and
// how many kernel launches that trace makes.
int resolve_kernel(int mode, uint64_t n_tuples);
// The stage-1 bounce cap a resident scene's staged launches use (its chosen pair's
// first cap, the built-in one while the choice is open).
uint32_t scene_stage_cap(const ResidentScene &rs);
// Both caps of the scene's chosen pair ({0, 0}, the built-in pair, while open).
StageCaps scene_stage_caps(const ResidentScene &rs);
// A staged call's caps under tuning state T: the chosen pair, or a device-timed trial
// of the next unmeasured candidate (trial >= 0; tune_end records its end).  The
// scene's first staged call runs untimed (it carries one-time costs).
StageCaps tune_begin(StageCapTune &T, int kernel_mode, const SceneConst &S, uint64_t n_pixels, uint32_t spp,
                     uint64_t chunk_budget, cudaStream_t s, int &trial);
void tune_end(StageCapTune &T, int trial, cudaStream_t s);
void tune_release(StageCapTune &T);
// gr_accumulate's tuning state for the scene's stone (created on first use).
StageCapTune &accum_tune(gr_ctx *ctx, const gr_scene *sc);
// The gr_accumulate tuning key of a scene (its stone, not its view).
uint64_t stone_key(const gr_scene *sc);
int trace_kernel_launches(int mode, const SceneConst &S, uint64_t n_tuples);
gr_status launch_fold(const float *xyz, uint32_t n_pixels, uint32_t spp, uint32_t first_pixel, float *film,
                      uint32_t kahan, cudaStream_t stream);
}  // namespace grh
