// gr_batch.cu -- gr_render_batch: many resident scenes in shared launches.
//
// The planner cuts every item (resident scene, film, sample range) into segments of
// whole pixels and packs them, grouped by scene class and in item order within a class,
// into launches of at most the context's per-launch tuple budget (chunk_budget / 12 B
// of per-tuple XYZ scratch); each launch runs the trace kernels specialised for its
// class (gr_batch_classes.cu), as the single-scene renders do.  Each launch
// is one k_trace_batch grid over all of its segments followed by one k_fold_batch
// grid, so scenes with few pixels or few samples share the device with the others
// instead of each paying a launch, a tail and a host round trip.  Per-tuple arithmetic
// and the per-pixel fold order are those of the single-scene kernels: every film is
// bit-identical to rendering its item alone with gr_render_resident.
//
// Launches are staged like the single-scene renders (gr_stage.cuh): k_trace_batch runs
// paths up to the stage cap and parks the survivors in their segment's park region,
// k_trace_batch_cont finishes them, one block per 128 parked paths of one segment.
//
// With GR_BATCH_GRAPH the launch sequence is captured once as a CUDA graph and
// replayed whenever the same batch shape recurs (same scenes, films, spp, frame sizes
// and tables); only the device tables, which carry the sample offsets, are uploaded
// again before each replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "gr_batch.cuh"
#include "gr_ctx.h"

using grh::fail;

namespace grd {
// The ordered per-pixel fold of a batched launch: one warp per pixel of each segment.
__global__ void k_fold_batch(const BatchSegment *__restrict__ segs, uint32_t n_segs) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const BatchSegment &G = segs[find_segment<1>(segs, n_segs, warp)];
    const uint64_t px = warp - G.warp_begin;
    if (px >= G.R.n_pixels) return;  // the grid's last warps past the final segment
    fold_pixel(G.xyz, px, G.R.spp, G.R.first_pixel + (uint32_t)px, G.film, G.kahan, G.cont, G.comp);
}
}  // namespace grd

namespace {

struct Launch {
    uint32_t seg_first, seg_count;
    uint64_t blocks, warps;
    uint32_t max_planes;
    bool extras;  // a segment's scene has frosted facets, scattering or a biaxial material
    uint64_t park_paths, park_blocks;  // park slots over the launch's segments, continuation blocks
    int K;        // the scene class of every segment (scene_class), -1: the extension kernels
};

struct Plan {
    std::vector<grd::SceneSlot> slots;
    std::vector<grd::BatchSegment> segs;
    std::vector<Launch> launches;
    uint64_t max_tuples = 0;  // scratch tuples one launch needs
    uint64_t max_park = 0;    // park slots one launch needs
    uint32_t max_segs = 0;    // segments of the largest launch (park slot counters)
};

// Park slots per launch: 1/16 of its tuples (paths alive after the stage cap are a few
// percent on the stones measured), at most 4 GiB of records; a segment whose region
// fills up finishes the rest of its paths in stage 1.
constexpr uint64_t kBatchParkLimit = (4ull << 30) / sizeof(grd::Path);

void place_park(Plan &P, Launch &L) {
    uint64_t tuples = 0;
    for (uint32_t i = 0; i < L.seg_count; ++i) tuples += P.segs[L.seg_first + i].R.n_tuples;
    const double scale = std::min(1.0 / 16.0, (double)kBatchParkLimit / (double)std::max<uint64_t>(tuples, 1));
    uint64_t off = 0, blocks = 0;
    for (uint32_t i = 0; i < L.seg_count; ++i) {
        grd::BatchSegment &g = P.segs[L.seg_first + i];
        uint64_t cap = (uint64_t)((double)g.R.n_tuples * scale) + 32;
        if (cap > g.R.n_tuples) cap = g.R.n_tuples;
        g.park_cap = (uint32_t)cap;
        g.park_off = off;
        g.park_block_begin = blocks;
        off += cap;
        blocks += (cap + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS;
    }
    L.park_paths = off;
    L.park_blocks = blocks;
    P.max_park = std::max(P.max_park, off);
    P.max_segs = std::max(P.max_segs, L.seg_count);
}

// Cuts the items into launches of at most `budget` tuples (a pixel whose spp alone
// exceeds the budget gets a launch of its own).  xyz pointers are offsets from 0
// until the scratch is placed.
gr_status make_plan(gr_ctx *ctx, const grh::BatchItem *items, uint32_t n_items, uint64_t budget, Plan &P) {
    std::unordered_map<uint64_t, uint32_t> slot_of;
    Launch cur{0, 0, 0, 0, 0, false, 0, 0, -1};
    uint64_t used = 0;
    auto close = [&]() {
        if (cur.seg_count) {
            place_park(P, cur);
            P.launches.push_back(cur);
        }
        P.max_tuples = std::max(P.max_tuples, used);
        cur = Launch{(uint32_t)P.segs.size(), 0, 0, 0, 0, false, 0, 0, -1};
        used = 0;
    };
    // Items grouped by scene class (stable within a class), so each launch runs the
    // kernels specialised for its class; unknown scenes fail in item order first.
    std::vector<int> cls(n_items, -1);
    for (uint32_t i = 0; i < n_items; ++i) {
        auto f = ctx->scenes.find(items[i].it.scene_id);
        if (f == ctx->scenes.end())
            return fail(GR_ENOTFOUND, "item %u: unknown scene id %llu", i, (unsigned long long)items[i].it.scene_id);
        cls[i] = grh::scene_class(f->second->S);
    }
    std::vector<uint32_t> order(n_items);
    for (uint32_t i = 0; i < n_items; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cls[a] < cls[b]; });
    for (uint32_t i : order) {
        const gr_batch_item &it = items[i].it;
        ResidentScene *rs = ctx->scenes.find(it.scene_id)->second;
        const uint64_t n_px = (uint64_t)rs->S.width * rs->S.height;
        if (it.spp == 0 || n_px == 0) continue;
        if (cur.seg_count && cur.K != cls[i]) close();  // one class per launch
        cur.K = cls[i];
        if (!it.film_device) return fail(GR_EINVAL, "item %u: film is NULL", i);
        if (rs->S.flags & GR_FLAG_FP64_RESOLVE)
            return fail(GR_EINVAL, "item %u: GR_FLAG_FP64_RESOLVE scenes render through the single-scene calls", i);
        auto sl = slot_of.find(it.scene_id);
        uint32_t slot;
        if (sl == slot_of.end()) {
            slot = (uint32_t)P.slots.size();
            grd::SceneSlot s;
            std::memset(&s, 0, sizeof(s));
            s.S = rs->S;
            s.B = resident_buffers(rs);
            P.slots.push_back(s);
            slot_of[it.scene_id] = slot;
        } else {
            slot = sl->second;
        }
        uint64_t next = 0;
        while (next < n_px) {
            uint64_t room = used < budget ? (budget - used) / it.spp : 0;
            if (room == 0) {
                if (used > 0) {
                    close();
                    cur.K = cls[i];
                    continue;
                }
                room = 1;
            }
            const uint64_t np = std::min(room, n_px - next);
            grd::BatchSegment g;
            std::memset(&g, 0, sizeof(g));
            g.R.first_pixel = (uint32_t)next;
            g.R.n_pixels = (uint32_t)np;
            g.R.sample_offset = it.sample_offset;
            g.R.spp = it.spp;
            g.R.n_tuples = np * it.spp;
            g.xyz = reinterpret_cast<float *>((uintptr_t)(3 * used * sizeof(float)));
            g.film = it.film_device;
            g.block_begin = cur.blocks;
            g.warp_begin = cur.warps;
            g.scene = slot;
            g.kahan = (rs->S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u;
            g.stage_cap = grh::scene_stage_cap(*rs);
            g.cont = items[i].cont;
            g.comp = items[i].comp;
            if (g.cont && g.kahan && !g.comp) return fail(GR_EINVAL, "item %u: continue mode with Kahan needs comp", i);
            P.segs.push_back(g);
            cur.seg_count++;
            cur.blocks += (g.R.n_tuples + grd::TRACE_THREADS - 1) / grd::TRACE_THREADS;
            cur.warps += np;
            cur.max_planes = std::max(cur.max_planes, rs->S.n_planes);
            cur.extras = cur.extras || grd::needs_extras(rs->S);
            used += g.R.n_tuples;
            next += np;
        }
    }
    close();
    return GR_OK;
}

// Capacity to reserve for `need` bytes: unchanged while it fits, else at least double
// the old capacity (and 1 MiB), capped at `limit` when that still covers `need`.  A
// regrowth frees the old buffer, which synchronises the device (and, for pinned
// memory, pins pages): geometric growth makes that rare in a long-running loop.
size_t grown(size_t cap, size_t need, size_t limit) {
    if (need <= cap) return need;
    size_t want = std::max<size_t>({need, 2 * cap, (size_t)1 << 20});
    if (want > limit) want = std::max(need, limit);
    return want;
}

gr_status launch_plan(const Plan &P, const grd::SceneSlot *slots, const grd::BatchSegment *segs, void *park_buf,
                      cudaStream_t s) {
    unsigned int *counts = (unsigned int *)park_buf;
    grd::Path *park = (grd::Path *)((char *)park_buf + (((size_t)P.max_segs * sizeof(unsigned int) + 255) & ~(size_t)255));
    for (const Launch &L : P.launches) {
        const size_t smem = grd::planes_smem_bytes(L.max_planes);
        GR_CUDA(cudaMemsetAsync(counts, 0, (size_t)L.seg_count * sizeof(unsigned int), s));
        if (L.extras) {
            grd::launch_batch_grids<true, grd::K_ANY, GR_TRACE_MIN_BLOCKS>(slots, segs + L.seg_first, L.seg_count, park,
                                                                           counts, L.blocks, L.park_blocks, smem, s);
        } else if (L.K >= 0) {
            const gr_status st = grh::launch_batch_class(L.K, slots, segs + L.seg_first, L.seg_count, park, counts,
                                                         L.blocks, L.park_blocks, smem, s);
            if (st != GR_OK) return st;
        } else {
            grd::launch_batch_grids<false, grd::K_ANY, GR_TRACE_MIN_BLOCKS>(slots, segs + L.seg_first, L.seg_count, park,
                                                                            counts, L.blocks, L.park_blocks, smem, s);
        }
        const unsigned T = 256;
        grd::k_fold_batch<<<(unsigned)((L.warps * 32 + T - 1) / T), T, 0, s>>>(segs + L.seg_first, L.seg_count);
    }
    GR_CUDA(cudaGetLastError());
    return GR_OK;
}

// The shape a captured graph is valid for: everything but the sample offsets.
std::vector<uint64_t> graph_key(const Plan &P, const void *tables, const void *xyz, const void *park) {
    std::vector<uint64_t> k;
    k.push_back((uint64_t)(uintptr_t)tables);
    k.push_back((uint64_t)(uintptr_t)xyz);
    k.push_back((uint64_t)(uintptr_t)park);
    k.push_back(P.max_segs);
    k.push_back(P.slots.size());
    for (const grd::BatchSegment &g : P.segs) {
        k.push_back((uint64_t)(uintptr_t)g.film);
        k.push_back(((uint64_t)g.R.first_pixel << 32) | g.R.n_pixels);
        k.push_back(((uint64_t)g.R.spp << 32) | g.scene);
        k.push_back((uint64_t)(uintptr_t)g.comp ^ g.cont);
    }
    for (const Launch &L : P.launches)
        k.push_back(((uint64_t)L.seg_count << 32) | L.max_planes | ((uint64_t)L.extras << 31) |
                    ((uint64_t)(uint8_t)(L.K + 1) << 20));
    return k;
}

}  // namespace

namespace grh {

gr_status batch_enqueue(gr_ctx *ctx, const BatchItem *items, uint32_t n_items, uint32_t flags, cudaStream_t stream) {
    uint64_t budget = ctx->chunk_budget / (3 * sizeof(float));
    if (budget > 0xFFFFFFFFull) budget = 0xFFFFFFFFull;  // tuple ids are u32 within a segment
    Plan P;
    gr_status st = make_plan(ctx, items, n_items, budget, P);
    if (st != GR_OK) return st;
    if (P.launches.empty()) return GR_OK;
    cudaStream_t s = stream ? stream : ctx->stream;

    st = ctx->xyz.reserve(grown(ctx->xyz.cap, (size_t)P.max_tuples * 3 * sizeof(float), ctx->chunk_budget));
    if (st != GR_OK) return st;
    const size_t slot_bytes = (P.slots.size() * sizeof(grd::SceneSlot) + 255) & ~(size_t)255;
    const size_t seg_bytes = P.segs.size() * sizeof(grd::BatchSegment);
    st = ctx->batch_tables.reserve(grown(ctx->batch_tables.cap, slot_bytes + seg_bytes, SIZE_MAX));
    if (st != GR_OK) return st;
    const size_t park_bytes = (((size_t)P.max_segs * sizeof(unsigned int) + 255) & ~(size_t)255) +
                              (size_t)P.max_park * sizeof(grd::Path);
    st = ctx->batch_park.reserve(grown(ctx->batch_park.cap, park_bytes, SIZE_MAX));
    if (st != GR_OK) return st;
    float *xyz = (float *)ctx->xyz.ptr;
    for (grd::BatchSegment &g : P.segs) g.xyz = xyz + ((uintptr_t)g.xyz) / sizeof(float);
    grd::SceneSlot *d_slots = (grd::SceneSlot *)ctx->batch_tables.ptr;
    grd::BatchSegment *d_segs = (grd::BatchSegment *)((char *)ctx->batch_tables.ptr + slot_bytes);
    // Stage both tables in the next pinned ring slot (once its previous upload has
    // been consumed) and upload them in one copy.  The device tables are shared by
    // every batch: stream order puts this copy after the previous batch's kernels.
    const int k = ctx->stage_next;
    ctx->stage_next = (k + 1) % gr_ctx::kStageSlots;
    if (ctx->stage_ev[k]) GR_CUDA(cudaEventSynchronize(ctx->stage_ev[k]));
    else GR_CUDA(cudaEventCreateWithFlags(&ctx->stage_ev[k], cudaEventDisableTiming));
    if (ctx->stage_cap[k] < slot_bytes + seg_bytes) {
        if (ctx->stage_host[k]) cudaFreeHost(ctx->stage_host[k]);
        ctx->stage_host[k] = nullptr;
        ctx->stage_cap[k] = 0;
        const size_t want = grown(ctx->stage_cap[k], slot_bytes + seg_bytes, SIZE_MAX);
        GR_CUDA(cudaHostAlloc(&ctx->stage_host[k], want, cudaHostAllocDefault));
        ctx->stage_cap[k] = want;
    }
    char *h = (char *)ctx->stage_host[k];
    std::memcpy(h, P.slots.data(), P.slots.size() * sizeof(grd::SceneSlot));
    std::memcpy(h + slot_bytes, P.segs.data(), seg_bytes);
    GR_CUDA(cudaMemcpyAsync(ctx->batch_tables.ptr, h, slot_bytes + seg_bytes, cudaMemcpyHostToDevice, s));
    GR_CUDA(cudaEventRecord(ctx->stage_ev[k], s));

    if (!(flags & GR_BATCH_GRAPH)) return launch_plan(P, d_slots, d_segs, ctx->batch_park.ptr, s);

    const std::vector<uint64_t> key = graph_key(P, ctx->batch_tables.ptr, ctx->xyz.ptr, ctx->batch_park.ptr);
    cudaGraphExec_t exec = nullptr;
    for (const BatchGraph &g : ctx->batch_graphs)
        if (g.key == key) exec = g.exec;
    if (!exec) {
        cudaGraph_t graph = nullptr;
        GR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        st = launch_plan(P, d_slots, d_segs, ctx->batch_park.ptr, s);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (st != GR_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return fail(GR_ECUDA, "batch graph capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(GR_ECUDA, "batch graph instantiation failed: %s", cudaGetErrorString(e));
        if (ctx->batch_graphs.size() >= kMaxBatchGraphs) {
            cudaGraphExecDestroy(ctx->batch_graphs.front().exec);
            ctx->batch_graphs.erase(ctx->batch_graphs.begin());
        }
        ctx->batch_graphs.push_back(BatchGraph{key, exec});
    }
    GR_CUDA(cudaGraphLaunch(exec, s));
    return GR_OK;
}

}  // namespace grh

// Items of at least this many path-samples render with the single-scene kernels (the
// stone's tuned schedule) instead of in a shared launch: one launch of ~2 M tuples
// already fills a B200 for many waves, and the specialised single-scene kernels at the
// stone's blocks-per-SM target run such a launch faster than the general batched
// kernels (measured on the c4 stones at full size: 577 M path-samples/s one stone at a
// time against 526 M packed).
#ifndef GR_BATCH_SOLO_MTUPLES
#define GR_BATCH_SOLO_MTUPLES 2
#endif

extern "C" gr_status gr_render_batch(gr_ctx *ctx, const gr_batch_item *items, uint32_t n_items, uint32_t flags,
                                     void *stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (n_items && !items) return fail(GR_EINVAL, "items is NULL");
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    std::vector<grh::BatchItem> packed;
    std::vector<std::pair<ResidentScene *, const gr_batch_item *>> solo;
    for (uint32_t i = 0; i < n_items; ++i) {
        const gr_batch_item &it = items[i];
        auto f = ctx->scenes.find(it.scene_id);
        if (f == ctx->scenes.end())
            return fail(GR_ENOTFOUND, "item %u: unknown scene id %llu", i, (unsigned long long)it.scene_id);
        ResidentScene *rs = f->second;
        const uint64_t tuples = (uint64_t)rs->S.width * rs->S.height * it.spp;
        if (tuples && !it.film_device) return fail(GR_EINVAL, "item %u: film is NULL", i);
        if (rs->S.flags & GR_FLAG_FP64_RESOLVE)
            return fail(GR_EINVAL, "item %u: GR_FLAG_FP64_RESOLVE scenes render through the single-scene calls", i);
        if (tuples >= ((uint64_t)GR_BATCH_SOLO_MTUPLES << 20))
            solo.emplace_back(rs, &it);
        else
            packed.push_back(grh::BatchItem{it, nullptr, 0u});
    }
    for (auto &p : solo) {
        const gr_status st = grh::render_resident_locked(ctx, p.first, p.second->sample_offset, p.second->spp,
                                                         p.second->film_device, s);
        if (st != GR_OK) return st;
    }
    return grh::batch_enqueue(ctx, packed.data(), (uint32_t)packed.size(), flags, s);
}
