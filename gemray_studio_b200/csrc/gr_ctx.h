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
// kBuiltinScheduleBlocks): a staged schedule.
struct StageCaps {
    uint32_t first = 0, second = 0;
    uint32_t blocks = 0;
};
// Blocks-per-SM targets the staged single-scene kernels are built for: register
// budgets of 56 / 48 / 40 / 32 per thread on 128-thread blocks (a target of 11 compiles
// to the same 40 registers as 12, 13-15 to the same 32 as 16).  Measured on B200, ms
// per frame at 9 / 10 / 12 / 16 blocks: the c2 brilliant (caps 12 / 20) 554.8 / 542.7 /
// 531.0 / 513.4, the c3 emerald (caps 8 / 16) 2019.6 / 1970.1 / 1937.1 / 1904.4 -- the
// latency of the scalar physics code is hidden better by more warps than it costs in
// spilled values.
constexpr int kScheduleBlockCount = 4;
constexpr uint32_t kScheduleBlocks[kScheduleBlockCount] = {9, 10, 12, 16};
// The blocks per SM of a staged launch whose schedule is still open.
constexpr uint32_t kBuiltinScheduleBlocks = 16;
// Stage-cap pairs a stone chooses between: the pair measured best on the c2 brilliant
// (long, TIR-trapped diamond paths), the one measured best on the c3 emerald (n ~ 1.6,
// shorter paths; 3.9% faster there) and a longer pair for longer paths still.
constexpr int kCapPairCount = 3;
constexpr uint32_t kCapPairs[kCapPairCount][2] = {{12, 20}, {8, 16}, {16, 28}};
// Candidate schedules: cap pair p at blocks b is candidate p * kScheduleBlockCount + b.
constexpr int kScheduleCandidates = kCapPairCount * kScheduleBlockCount;
inline StageCaps schedule_candidate(int c) {
    return StageCaps{kCapPairs[c / kScheduleBlockCount][0], kCapPairs[c / kScheduleBlockCount][1],
                     kScheduleBlocks[c % kScheduleBlockCount]};
}
// The candidate index of a schedule, -1 if it is not one.
inline int schedule_index(uint32_t first, uint32_t second, uint32_t blocks) {
    for (int c = 0; c < kScheduleCandidates; ++c) {
        const StageCaps k = schedule_candidate(c);
        if (k.first == first && k.second == second && k.blocks == blocks) return c;
    }
    return -1;
}

// The staged schedule (stage caps and blocks per SM) a stone's staged renders use.
// Every schedule gives the same films, but the fastest depends on the stone's path
// lengths and register pressure.  From the stone's second staged call on, calls are
// timed on the device as trials (the whole call: its chunks cover different parts of
// the image), in two rounds: the first cap pair at each blocks-per-SM target, then the
// other pairs at the fastest target; the candidate with the least time per tuple is
// kept.  A choice can also come from the context's tuning table (measured earlier for
// the same stone on this device, gr_tuning_load) or be pinned (gr_scene_set_schedule).
struct StageCapTune {
    static constexpr int kTrials = kScheduleBlockCount + kCapPairCount - 1;
    uint64_t key = 0;           // the stone (stone_key), for the context's tuning table
    int best = -1;              // chosen candidate, -1 while measuring
    uint32_t staged_calls = 0;  // staged calls seen
    int n_trials = 0;           // trials issued
    float ms_per_mtuple[kScheduleCandidates];
    struct Trial {
        cudaEvent_t start = nullptr, stop = nullptr;
        int candidate = 0;
        uint64_t tuples = 0;
        bool ended = false;  // stop recorded (tune_end): until then the trial is not read
        bool done = false;
    } trial[kTrials];
    StageCapTune() {
        for (float &m : ms_per_mtuple) m = 3.0e38f;  // unmeasured: never chosen over a measured one
    }
};

// A schedule chosen for a stone on this context's device: the tuning table's entry.
struct TunedSchedule {
    int candidate = 0;
    float ms_per_mtuple = 0.0f;
};

struct ResidentScene {
    SceneConst S;
    uint64_t stone = 0;  // stone_key of the uploaded scene
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
    // depth, flags -- what sets the path lengths -- and the environment kind, which
    // selects the kernels); cleared past kMaxAccumTunes stones
    std::map<uint64_t, StageCapTune> accum_tune;
    static constexpr size_t kMaxAccumTunes = 64;
    // Schedules chosen per stone on this device (measured here, or read from a tuning
    // table by gr_tuning_load): a stone met again starts from its entry, without trials.
    std::map<uint64_t, TunedSchedule> tuned;
    std::string tuning_cache;  // GR_TUNING_CACHE at creation: loaded then, saved at gr_destroy
    size_t trace_used = 0, fold_used = 0;
    uint64_t trace_launches = 0, fold_launches = 0;
    // gr_render_batch: scene-slot + segment tables, captured launch sequences, and a
    // ring of pinned host staging buffers for the table uploads (a pageable source
    // would make each upload wait for the previous batch to reach its copy)
    grh::DeviceBuffer batch_tables, batch_park;  // segment tables; staged park records + slot counters
    // gr_accumulate's pinned readback buffer (grown, kept)
    void *host_stage = nullptr;
    size_t host_stage_cap = 0;
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
// gr_render_resident's body (the stone's tuned schedule, its trials included); the
// caller holds ctx->mu and has made ctx->device current.
gr_status render_resident_locked(gr_ctx *ctx, ResidentScene *rs, uint32_t sample_offset, uint32_t spp, float *film_dev,
                                 cudaStream_t s);
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
struct SceneSlot;
struct BatchSegment;
}
namespace grh {
// The two trace grids of a batched launch whose segments all have scene class K
// (gr_batch_classes.cu); K is a clear-isotropic or general class with its environment.
gr_status launch_batch_class(int K, const grd::SceneSlot *slots, const grd::BatchSegment *segs, uint32_t n_segs,
                             grd::Path *park, unsigned int *counts, uint64_t blocks, uint64_t park_blocks, size_t smem,
                             cudaStream_t s);
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
    uint32_t blocks;  // kScheduleBlocks entry, 0 = kBuiltinScheduleBlocks
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
// The scene's chosen schedule ({0, 0, 0}, the built-in one, while open).
StageCaps scene_stage_caps(const ResidentScene &rs);
// A staged call's schedule under tuning state T: the chosen one, or a device-timed
// trial of the next candidate (trial >= 0; tune_end records its end).  The stone's
// first staged call runs untimed (it carries one-time costs).  A finished choice is
// entered in ctx->tuned.  The caller holds ctx->mu.
StageCaps tune_begin(gr_ctx *ctx, StageCapTune &T, const SceneConst &S, uint64_t n_pixels, uint32_t spp,
                     cudaStream_t s, int &trial);
// The caller holds ctx->mu (a trial is read only after its end is recorded).
void tune_end(StageCapTune &T, int trial, cudaStream_t s);
// Reads T's finished trials; chooses (and enters the choice in ctx->tuned) once all
// are in.  The caller holds ctx->mu.
void tune_harvest(gr_ctx *ctx, StageCapTune &T);
// A fresh tuning state for stone `key`, starting from ctx->tuned's entry if any.
void tune_init(gr_ctx *ctx, StageCapTune &T, uint64_t key);
void tune_release(StageCapTune &T);
// gr_accumulate's tuning state for the scene's stone (created on first use).
StageCapTune &accum_tune(gr_ctx *ctx, const gr_scene *sc);
// The gr_accumulate tuning key of a scene (its stone, not its view).
uint64_t stone_key(const gr_scene *sc);
int trace_kernel_launches(int mode, const SceneConst &S, uint64_t n_tuples);
// Park slots of a staged launch's first stage (1/8 of its tuples, at least 1,024, at
// most 4 GiB of records), and the park buffer bytes of both capped stages.
uint64_t staged_park_slots(uint64_t n_tuples);
size_t staged_park_bytes(uint64_t n_tuples);
gr_status launch_fold(const float *xyz, uint32_t n_pixels, uint32_t spp, uint32_t first_pixel, float *film,
                      uint32_t kahan, cudaStream_t stream);
}  // namespace grh
