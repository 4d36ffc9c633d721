// gr_serve.cu -- the render-request loop: gr_submit / gr_poll / gr_wait / gr_cancel.
//
// Requests mirror RenderRequest{request_id, first_sample, samples}
// (crates/gemray-net/src/messages/render.rs:65-70) over resident scenes.  A worker
// thread per context runs continuous batching:
//   * admission -- queued requests are admitted in arrival order while their film
//     fits the context's device-memory budget next to the resident scenes and the
//     films of running requests; a film is allocated and zeroed on admission;
//   * ticks -- each tick is ONE batched launch (gr_batch.cu) filled from the running
//     renders in arrival order, each contributing all of its remaining samples until
//     the tick's tuple budget is spent, so small requests finish in a single tick and
//     share it with others; one tick is in flight at a time;
//   * retirement -- when a tick's event completes its slices count as folded;
//     a render is DONE when all its samples are; cancellation takes effect between
//     slices;
//   * metric requests (pose sweeps) skip admission (they hold no film): a second
//     thread runs them in arrival order on its own high-priority stream, beside the
//     tick in flight, so a sweep neither waits for a tick nor holds one up;
//   * render lanes -- a render without a slice size of its own (slice_spp == 0) is
//     not cut into ticks but into chunks of whole pixels over its whole sample range
//     (GR_SERVE_CHUNK_MTUPLES path-samples), rendered with the single-scene kernels
//     and the stone's tuned schedule (the kernels and schedule of gr_render_resident)
//     on a lane's own stream, with scratch of its own.  After each chunk the lane takes
//     the next chunk of whichever admitted render comes first by submission time plus
//     remaining work: a short request passes a long one that has not waited or run
//     long, so it waits at most about a chunk behind it, while a long one that has
//     waited longer than a newer request's remaining work goes first.  Cancellation takes effect
//     between chunks and leaves a zero film.  GR_SERVE_POLICY=0 selects size-class
//     lanes instead (each request whole on a lane of its size class, smaller classes
//     at higher stream priority, several requests on the device at once).  Sliced
//     renders (slice_spp > 0, progressive rendering) go to the ticks.
// Slices fold in continue mode (fold_pixel): each slice carries the pixel's running
// sum on from the film (and the Kahan compensation from a side buffer), and a request
// starts on a zero film, so its film is one sequential per-pixel sum over all of its
// samples -- bit-identical to one gr_render_resident call over the same sample range
// on a zero film, whatever the slicing and whatever else is running.  Slices are
// therefore sized freely by the scheduler.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gr_ctx.h"
#include "gr_launch.cuh"

using grh::fail;

namespace {

using Clock = std::chrono::steady_clock;

// A request's film (or Kahan compensation) from the stream-ordered allocator: taking
// and returning it never synchronises the device, so admissions and releases do not
// stall the ticks in flight.  Films come from the serve loop's own pool, which keeps
// the memory it has mapped (release threshold = the serve budget): the default pool
// gives its free memory back at every synchronisation, and mapping it again on the
// next admission was measured at 10-380 ms on B200 -- time the worker, which admits
// under the serve lock, spent stalled with the ticks and every submitter behind it.
struct StreamBuffer {
    void *ptr = nullptr;
    cudaError_t alloc(size_t bytes, cudaStream_t s, cudaMemPool_t pool) {
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&ptr, bytes, pool, s) : cudaMallocAsync(&ptr, bytes, s);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return e;
        }
        return cudaMemsetAsync(ptr, 0, bytes, s);
    }
    void release(cudaStream_t s) {
        if (ptr) cudaFreeAsync(ptr, s);
        ptr = nullptr;
    }
};

struct Request {
    uint64_t id = 0;
    gr_request r{};
    std::vector<gr_pose> poses;          // metrics
    std::vector<gr_plane> planes;        // metrics
    gr_material material{};              // metrics
    std::vector<gr_metrics_out> metrics; // metrics results
    uint32_t state = GR_REQ_QUEUED;
    gr_status error = GR_OK;
    uint64_t film_bytes = 0;     // film (+ Kahan compensation) bytes held on the device
    uint64_t n_px = 0;
    bool kahan = false;
    StreamBuffer film, comp;
    uint32_t issued = 0, done = 0, in_flight = 0;  // samples per pixel
    uint64_t px_done = 0;      // lane renders: pixels whose samples are all folded
    uint64_t px_issued = 0;    // policy 1: pixels whose chunk has been queued
    uint64_t px_inflight = 0;  // policy 1: pixels of queued chunks not yet retired
    cudaEvent_t film_ev = nullptr;  // policy 1: the film's allocation and zeroing, for other lanes' streams
    bool cancel = false;
    int lane_class = -1;  // rendered whole by a lane of this size class; -1: in ticks
    bool admitted = false;  // film_bytes counted in the serve budget
    Clock::time_point t_submit, t_admit, t_done;
};

// Path-samples one tick carries: ~10-30 ms of transport on B200, the latency quantum
// of the request loop (a new arrival joins the tick after the one in flight).
#ifndef GR_SERVE_TICK_MTUPLES
#define GR_SERVE_TICK_MTUPLES 8
#endif
constexpr uint64_t kTickTuples = (uint64_t)GR_SERVE_TICK_MTUPLES << 20;
// Slice order within a tick: 0 = arrival order, 1 = least remaining work first.
#ifndef GR_SERVE_ORDER
#define GR_SERVE_ORDER 0
#endif
// 1: while several renders are active none takes more than half of a tick.
#ifndef GR_SERVE_HALF_CAP
#define GR_SERVE_HALF_CAP 1
#endif
// Ticks queued on the device at once.  One: the host plans the next tick in ~0.1 ms,
// so a second tick in flight buys no throughput and would make an arrival wait
// behind two ticks instead of one.
constexpr size_t kTicksInFlight = 1;
// Film pool memory mapped when the serve loop starts (at most the serve budget), so
// admissions map no memory until the live films pass it (~2,800 films of 384^2
// pixels with Kahan compensation); growing the pool was measured at up to ~0.5 s.
constexpr uint64_t kFilmPoolReserve = 4ull << 30;
// Render lanes by size class: path-samples up to GR_SERVE_SMALL_MTUPLES M, up to
// GR_SERVE_BULK_MTUPLES M, and larger; lanes per class; a lane's chunk (scratch) size.
#ifndef GR_SERVE_SMALL_MTUPLES
#define GR_SERVE_SMALL_MTUPLES 2
#endif
#ifndef GR_SERVE_BULK_MTUPLES
#define GR_SERVE_BULK_MTUPLES GR_SERVE_TICK_MTUPLES
#endif
// Stream priorities of the classes: 0 = the smaller the request, the higher its
// priority; 1 = the larger, the higher.
#ifndef GR_SERVE_LANE_ORDER
#define GR_SERVE_LANE_ORDER 0
#endif
// Lane policy: 0 = size classes, each request rendered whole by a lane of its class;
// 1 = one shared queue of chunks: a lane renders GR_SERVE_CHUNK_MTUPLES path-samples
// (whole pixels) of the request that comes first in the order "submission time +
// remaining work at GR_SERVE_PS_PER_TUPLE picoseconds per path-sample", then chooses
// again, with up to GR_SERVE_CHUNK_DEPTH chunks queued on its stream (a second one
// hides the host's turn between chunks but makes a new arrival wait behind two).  The
// order lets a short request pass a long one that has not waited or run long, and puts
// a long one that has ahead of newer short ones (GR_SERVE_PS_PER_TUPLE 0: oldest first;
// very large: least remaining work first).  The defaults are the measured best on B200
// for the c5 request stream (served p99 against a serial server's): 16 M path-sample
// chunks, one queued, 0.7 ns per path-sample.
#ifndef GR_SERVE_POLICY
#define GR_SERVE_POLICY 1
#endif
#ifndef GR_SERVE_CHUNK_MTUPLES
#define GR_SERVE_CHUNK_MTUPLES 16
#endif
#ifndef GR_SERVE_CHUNK_LANES
#define GR_SERVE_CHUNK_LANES 1
#endif
#ifndef GR_SERVE_PS_PER_TUPLE
#define GR_SERVE_PS_PER_TUPLE 700
#endif
#ifndef GR_SERVE_CHUNK_DEPTH
#define GR_SERVE_CHUNK_DEPTH 1
#endif
constexpr size_t kChunksInFlight = GR_SERVE_CHUNK_DEPTH;
constexpr int kLaneClasses = 3;
constexpr uint32_t kLanesPerClass[kLaneClasses] = {2, 1, 1};
constexpr uint64_t kClassTuples[kLaneClasses] = {(uint64_t)GR_SERVE_SMALL_MTUPLES << 20,
                                                 (uint64_t)GR_SERVE_BULK_MTUPLES << 20, 22ull << 20};

int lane_class(uint64_t tuples) {
    return tuples <= kClassTuples[0] ? 0 : tuples <= kClassTuples[1] ? 1 : 2;
}

struct Tick {
    cudaEvent_t ev = nullptr;
    std::vector<std::pair<uint64_t, uint32_t>> slices;  // (request id, spp)
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

struct ServeState {
    std::mutex mu;
    cudaStream_t metrics_stream = nullptr;  // metric sweeps, beside the ticks
    struct Lane {
        int cls = 0;
        cudaStream_t stream = nullptr;
        grh::DeviceBuffer xyz, park;  // a chunk's per-tuple XYZ and park records
        std::thread th;
    };
    std::vector<Lane *> lanes;
    std::condition_variable cv_lane;
    std::deque<uint64_t> lane_queue[kLaneClasses];  // admitted lane renders per class, admission order
    std::vector<uint64_t> lane_pending;  // policy 1: admitted lane renders not yet finished
    cudaMemPool_t film_pool = nullptr;      // request films (null: the device's default pool)
    std::condition_variable cv_work, cv_done, cv_metrics;
    std::unordered_map<uint64_t, Request *> reqs;
    std::deque<uint64_t> queue;   // renders, admission order
    std::deque<uint64_t> metric_queue;  // metric sweeps, arrival order
    std::vector<uint64_t> running;
    uint64_t next_id = 1;
    uint64_t film_bytes = 0;      // films of admitted requests
    bool stop = false;
    std::thread worker, metrics_worker;
};

namespace {

void finish(ServeState &sv, Request *q, uint32_t state, gr_status err = GR_OK) {
    q->state = state;
    q->error = err;
    q->t_done = Clock::now();
    if (q->t_admit.time_since_epoch().count() == 0) q->t_admit = q->t_done;  // ended while queued
    sv.cv_done.notify_all();
}

// Admission in arrival order while films fit the budget (caller holds sv.mu).
void admit(gr_ctx *ctx, ServeState &sv, uint64_t resident_bytes) {
    while (!sv.queue.empty()) {
        Request *q = sv.reqs[sv.queue.front()];
        if (q->cancel) {
            sv.queue.pop_front();
            finish(sv, q, GR_REQ_CANCELLED);
            continue;
        }
        if (resident_bytes + q->film_bytes > ctx->serve_budget) {  // can never fit, even with no other film
            sv.queue.pop_front();
            finish(sv, q, GR_REQ_FAILED, GR_EBUSY);
            continue;
        }
        if (resident_bytes + sv.film_bytes + q->film_bytes > ctx->serve_budget) break;  // wait for releases
        if (!sv.lanes.empty() && q->r.slice_spp == 0) {
            // a lane renders it whole; the lane takes the film on its own stream
            sv.queue.pop_front();
            sv.film_bytes += q->film_bytes;
            q->admitted = true;
            q->state = GR_REQ_RUNNING;
            q->t_admit = Clock::now();
            q->lane_class = lane_class((uint64_t)q->r.spp * q->n_px);
            if (GR_SERVE_POLICY == 1)
                sv.lane_pending.push_back(q->id);
            else
                sv.lane_queue[q->lane_class].push_back(q->id);
            sv.cv_lane.notify_all();
            continue;
        }
        const size_t fb = (size_t)q->n_px * 3 * sizeof(float);
        if (q->film.alloc(fb, ctx->stream, sv.film_pool) != cudaSuccess ||
            (q->kahan && q->comp.alloc(fb, ctx->stream, sv.film_pool) != cudaSuccess)) {
            sv.queue.pop_front();
            q->film.release(ctx->stream);
            q->comp.release(ctx->stream);
            finish(sv, q, GR_REQ_FAILED, GR_ENOMEM);
            continue;
        }
        sv.queue.pop_front();
        sv.film_bytes += q->film_bytes;
        q->admitted = true;
        q->state = GR_REQ_RUNNING;
        q->t_admit = Clock::now();
        sv.running.push_back(q->id);
    }
}

// One chunk of a lane render: pixels [first, first + count) of request q over its whole
// sample range, traced with the single-scene kernels (the stone's tuned schedule,
// which lane chunks help choose like gr_render_resident calls; never the sorted
// kernel, whose blocks stay resident until its launch ends) and folded in add mode onto
// its film, on the lane's stream; returns after the stream has drained.  The first
// chunk takes the zero film from the loop's pool on the lane's stream.  The scene is
// marked in use meanwhile, so it cannot be released under the launches.
gr_status lane_chunk(gr_ctx *ctx, ServeState *sv, ServeState::Lane *lane, Request *q, uint64_t first, uint64_t count) {
    const uint32_t spp = q->r.spp;
    gr_status st = GR_OK;
    if (!q->film.ptr && q->film.alloc((size_t)q->n_px * 3 * sizeof(float), lane->stream, sv->film_pool) != cudaSuccess) {
        cudaGetLastError();
        return GR_ENOMEM;
    }
    SceneConst S;
    grd::SceneBuffers B;
    StageCaps caps;
    int mode = GR_KERNEL_AUTO;
    int trial = -1;
    ResidentScene *rs = nullptr;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->scenes.find(q->r.scene_id);
        if (it == ctx->scenes.end()) return GR_ENOTFOUND;
        rs = it->second;
        rs->users++;
        S = rs->S;
        B = resident_buffers(rs);
        if (ctx->kernel_mode != GR_KERNEL_SORTED) mode = ctx->kernel_mode;
        caps = grh::tune_begin(ctx, rs->tune, S, count, spp, lane->stream, trial);
    }
    const uint64_t step_px = std::max<uint64_t>(1, std::min<uint64_t>(count, kClassTuples[2] / spp));
    st = lane->xyz.reserve((size_t)step_px * spp * 12);
    for (uint64_t p = first; st == GR_OK && p < first + count; p += step_px) {
        if (q->cancel) break;  // between launches
        grd::LaunchRange R;
        R.first_pixel = (uint32_t)p;
        R.n_pixels = (uint32_t)std::min<uint64_t>(step_px, first + count - p);
        R.sample_offset = q->r.sample_offset;
        R.spp = spp;
        R.n_tuples = (uint64_t)R.n_pixels * spp;
        st = grh::launch_trace(ctx, S, B, R, (float *)lane->xyz.ptr, lane->stream, mode, &lane->park, caps);
        if (st == GR_OK)
            st = grh::launch_fold((const float *)lane->xyz.ptr, R.n_pixels, spp, R.first_pixel, (float *)q->film.ptr,
                                  (S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u, lane->stream);
    }
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        grh::tune_end(rs->tune, trial, lane->stream);
    }
    if (cudaStreamSynchronize(lane->stream) != cudaSuccess && st == GR_OK) st = GR_ECUDA;
    std::lock_guard<std::mutex> lk(ctx->mu);
    rs->users--;
    return st;
}

// Ends a lane render (caller holds sv->mu).  A cancelled one keeps no samples: its film,
// if it has one, is zeroed on the lane's stream first.
void lane_finish(ServeState *sv, ServeState::Lane *lane, Request *q, gr_status st) {
    q->in_flight = 0;
    if (st != GR_OK) {
        finish(*sv, q, GR_REQ_FAILED, st);
    } else if (q->cancel) {
        if (q->film.ptr) {
            cudaMemsetAsync(q->film.ptr, 0, (size_t)q->n_px * 3 * sizeof(float), lane->stream);
            cudaStreamSynchronize(lane->stream);
        }
        finish(*sv, q, GR_REQ_CANCELLED);
    } else {
        q->done = q->r.spp;
        finish(*sv, q, GR_REQ_DONE);
    }
}

// Policy 1: the pending render whose next chunk comes first (submission time + remaining
// work), or -1 when none has pixels left to queue (caller holds sv->mu).
int next_chunk_owner(ServeState &sv) {
    int pick = -1;
    uint64_t best = UINT64_MAX;
    for (size_t i = 0; i < sv.lane_pending.size(); ++i) {
        const Request *c = sv.reqs[sv.lane_pending[i]];
        if (c->cancel || c->px_issued >= c->n_px) continue;
        const uint64_t left = (c->n_px - c->px_issued) * c->r.spp;
        const uint64_t key = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                                 c->t_submit.time_since_epoch()).count() +
                             left * (uint64_t)GR_SERVE_PS_PER_TUPLE / 1000;
        if (key < best) {
            best = key;
            pick = (int)i;
        }
    }
    return pick;
}

// Policy 1: a cancelled pending render with no chunk queued, or -1 (caller holds sv->mu).
int idle_cancelled(ServeState &sv) {
    for (size_t i = 0; i < sv.lane_pending.size(); ++i) {
        const Request *c = sv.reqs[sv.lane_pending[i]];
        if (c->cancel && c->px_inflight == 0) return (int)i;
    }
    return -1;
}

// Policy 1: queue one chunk of q on the lane's stream (no wait).  The first chunk takes
// the film (zeroed, stream-ordered) and records film_ev, which later chunks on any
// lane's stream wait for; the scene stays in use until the chunk retires (*rs_out).
gr_status lane_launch(gr_ctx *ctx, ServeState::Lane *lane, Request *q, uint64_t first, uint64_t count,
                      ResidentScene **rs_out) {
    *rs_out = nullptr;
    const uint32_t spp = q->r.spp;
    if (q->film_ev) GR_CUDA(cudaStreamWaitEvent(lane->stream, q->film_ev, 0));
    SceneConst S;
    grd::SceneBuffers B;
    StageCaps caps;
    int mode = GR_KERNEL_AUTO;
    int trial = -1;
    ResidentScene *rs = nullptr;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->scenes.find(q->r.scene_id);
        if (it == ctx->scenes.end()) return GR_ENOTFOUND;
        rs = it->second;
        rs->users++;
        *rs_out = rs;
        S = rs->S;
        B = resident_buffers(rs);
        if (ctx->kernel_mode != GR_KERNEL_SORTED) mode = ctx->kernel_mode;
        caps = grh::tune_begin(ctx, rs->tune, S, count, spp, lane->stream, trial);
    }
    gr_status st = lane->xyz.reserve((size_t)count * spp * 12);
    grd::LaunchRange R;
    R.first_pixel = (uint32_t)first;
    R.n_pixels = (uint32_t)count;
    R.sample_offset = q->r.sample_offset;
    R.spp = spp;
    R.n_tuples = (uint64_t)count * spp;
    if (st == GR_OK) st = grh::launch_trace(ctx, S, B, R, (float *)lane->xyz.ptr, lane->stream, mode, &lane->park, caps);
    if (st == GR_OK)
        st = grh::launch_fold((const float *)lane->xyz.ptr, R.n_pixels, spp, R.first_pixel, (float *)q->film.ptr,
                              (S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u, lane->stream);
    std::lock_guard<std::mutex> lk(ctx->mu);
    grh::tune_end(rs->tune, trial, lane->stream);
    return st;
}

// A render lane.  Policy 0: the admitted renders of the lane's size class, one at a
// time, each rendered whole (in chunks of the class's size).  Policy 1: chunks of the
// pending renders in the order of next_chunk_owner, up to kChunksInFlight queued on the
// lane's stream; a request finishes when its last chunk retires (or, cancelled, when
// its queued chunks have retired).
void lane_main(gr_ctx *ctx, ServeState *sv, ServeState::Lane *lane) {
    cudaSetDevice(ctx->device);
    if (GR_SERVE_POLICY == 1) {
        struct Flight {
            Request *q;
            uint64_t first, count;
            ResidentScene *rs;
            gr_status st;
            cudaEvent_t ev;
        };
        std::deque<Flight> flight;
        std::vector<cudaEvent_t> spare;
        const uint64_t chunk_tuples = (uint64_t)GR_SERVE_CHUNK_MTUPLES << 20;
        for (;;) {
            Request *q = nullptr;
            uint64_t first = 0, count = 0;
            gr_status st = GR_OK;
            {
                std::unique_lock<std::mutex> lk(sv->mu);
                if (flight.empty()) {
                    sv->cv_lane.wait(lk, [&] {
                        return sv->stop || next_chunk_owner(*sv) >= 0 || idle_cancelled(*sv) >= 0;
                    });
                    for (int c; (c = idle_cancelled(*sv)) >= 0;) {  // cancelled before (or between) chunks
                        Request *r = sv->reqs[sv->lane_pending[c]];
                        sv->lane_pending.erase(sv->lane_pending.begin() + c);
                        lane_finish(sv, lane, r, r->error);
                    }
                    if (next_chunk_owner(*sv) < 0) {
                        if (sv->stop) return;  // stopping, nothing left to queue
                        continue;
                    }
                }
                const int i = flight.size() < kChunksInFlight ? next_chunk_owner(*sv) : -1;
                if (i >= 0) {
                    q = sv->reqs[sv->lane_pending[i]];
                    first = q->px_issued;
                    const uint64_t left = q->n_px - first;
                    count = std::min<uint64_t>(std::max<uint64_t>(1, chunk_tuples / q->r.spp), left);
                    // a remainder under half a chunk joins this one while the lane's
                    // scratch holds both: a short last launch costs its own stage tails
                    if (2 * (left - count) * q->r.spp <= chunk_tuples && left * q->r.spp <= kClassTuples[2])
                        count = left;
                    q->px_issued += count;
                    q->px_inflight += count;
                    q->issued = q->in_flight = q->r.spp;
                    if (!q->film.ptr) {  // the first chunk: the zero film, then its event
                        if (q->film.alloc((size_t)q->n_px * 3 * sizeof(float), lane->stream, sv->film_pool) !=
                                cudaSuccess ||
                            cudaEventCreateWithFlags(&q->film_ev, cudaEventDisableTiming) != cudaSuccess ||
                            cudaEventRecord(q->film_ev, lane->stream) != cudaSuccess) {
                            cudaGetLastError();
                            st = GR_ENOMEM;
                        }
                    }
                }
            }
            if (q) {
                Flight f{q, first, count, nullptr, st, nullptr};
                if (f.st == GR_OK) f.st = lane_launch(ctx, lane, q, first, count, &f.rs);
                if (!spare.empty()) {
                    f.ev = spare.back();
                    spare.pop_back();
                } else if (cudaEventCreateWithFlags(&f.ev, cudaEventDisableTiming) != cudaSuccess) {
                    f.ev = nullptr;
                }
                if (f.ev && cudaEventRecord(f.ev, lane->stream) != cudaSuccess && f.st == GR_OK) f.st = GR_ECUDA;
                flight.push_back(f);
                continue;  // fill the pipeline
            }
            // the pipeline is full, or nothing is left to queue: retire the oldest chunk
            Flight f = flight.front();
            flight.pop_front();
            cudaError_t e = f.ev ? cudaEventSynchronize(f.ev) : cudaStreamSynchronize(lane->stream);
            if (e != cudaSuccess && f.st == GR_OK) f.st = GR_ECUDA;
            if (f.ev) spare.push_back(f.ev);
            if (f.rs) {
                std::lock_guard<std::mutex> lk(ctx->mu);
                f.rs->users--;
            }
            std::lock_guard<std::mutex> lk(sv->mu);
            Request *r = f.q;
            r->px_inflight -= f.count;
            if (f.st == GR_OK) r->px_done += f.count;
            if (f.st != GR_OK && r->error == GR_OK) {
                r->error = f.st;
                r->cancel = true;  // queue no more of it
            }
            if (r->px_inflight == 0 && (r->cancel || r->px_done == r->n_px)) {
                auto &pend = sv->lane_pending;
                pend.erase(std::remove(pend.begin(), pend.end(), r->id), pend.end());
                lane_finish(sv, lane, r, r->error);
            }
            sv->cv_lane.notify_all();
        }
    }
    for (;;) {
        Request *q = nullptr;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            auto &queue = sv->lane_queue[lane->cls];
            sv->cv_lane.wait(lk, [&] { return sv->stop || !queue.empty(); });
            if (queue.empty()) return;  // stopping, nothing left
            q = sv->reqs[queue.front()];
            queue.pop_front();
            if (q->cancel) {
                lane_finish(sv, lane, q, GR_OK);
                continue;
            }
            q->issued = q->in_flight = q->r.spp;
        }
        gr_status st = GR_OK;
        const uint64_t chunk_px = std::max<uint64_t>(1, kClassTuples[lane->cls] / q->r.spp);
        for (uint64_t p = 0; st == GR_OK && p < q->n_px && !q->cancel; p += chunk_px)
            st = lane_chunk(ctx, sv, lane, q, p, std::min<uint64_t>(chunk_px, q->n_px - p));
        std::lock_guard<std::mutex> lk(sv->mu);
        q->px_done = q->n_px;
        lane_finish(sv, lane, q, st);
    }
}

void worker_main(gr_ctx *ctx, ServeState *sv) {
    cudaSetDevice(ctx->device);
    std::deque<Tick> flight;
    std::vector<cudaEvent_t> spare;
    auto retire = [&](Tick &t) {  // caller holds sv->mu; the tick's event has completed
        for (auto &s : t.slices) {
            auto it = sv->reqs.find(s.first);
            if (it == sv->reqs.end()) continue;
            Request *q = it->second;
            q->in_flight -= s.second;
            q->done += s.second;
        }
        spare.push_back(t.ev);
    };
    for (;;) {
        // 1. retire finished ticks (always the oldest first: ticks complete in order)
        while (!flight.empty()) {
            const bool must_wait = flight.size() >= kTicksInFlight;
            cudaError_t e = must_wait ? cudaEventSynchronize(flight.front().ev) : cudaEventQuery(flight.front().ev);
            if (e == cudaErrorNotReady) break;
            std::lock_guard<std::mutex> lk(sv->mu);
            retire(flight.front());
            flight.pop_front();
        }
        std::vector<grh::BatchItem> items;
        std::vector<std::pair<uint64_t, uint32_t>> slices;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            // 2. completions and cancellations of running requests
            std::vector<uint64_t> keep;
            for (uint64_t id : sv->running) {
                Request *q = sv->reqs[id];
                if (q->r.kind == GR_REQ_RENDER && q->in_flight == 0 && (q->cancel || q->done >= q->r.spp)) {
                    finish(*sv, q, q->done >= q->r.spp ? GR_REQ_DONE : GR_REQ_CANCELLED);
                    continue;
                }
                keep.push_back(id);
            }
            sv->running.swap(keep);
            // 3. admission (resident_bytes is read without ctx->mu: a stale value only
            //    delays or advances an admission by one tick)
            admit(ctx, *sv, ctx->resident_bytes);
            // 4. this tick's slices: running requests in arrival order, each taking all of
            //    its remaining samples until the tick's tuple budget is spent (no single
            //    request more than half of it while others wait); a fixed slice_spp caps
            //    a request's share per tick instead
            uint32_t n_active = 0;
            for (uint64_t id : sv->running) {
                Request *q = sv->reqs[id];
                n_active += q->r.kind == GR_REQ_RENDER && !q->cancel && q->issued < q->r.spp;
            }
            const uint64_t cap = GR_SERVE_HALF_CAP && n_active > 1 ? kTickTuples / 2 : kTickTuples;
            uint64_t budget = kTickTuples;
            std::vector<uint64_t> order(sv->running);
            if (GR_SERVE_ORDER == 1) {
                auto left = [&](uint64_t id) {
                    const Request *q = sv->reqs[id];
                    return q->r.kind == GR_REQ_RENDER ? (uint64_t)(q->r.spp - q->issued) * q->n_px : 0;
                };
                std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return left(a) < left(b); });
            }
            for (uint64_t id : order) {
                Request *q = sv->reqs[id];
                if (q->cancel || q->issued >= q->r.spp) continue;
                const uint64_t px = std::max<uint64_t>(1, q->n_px);
                uint64_t want = std::min(budget, cap) / px;
                if (want == 0) {
                    if (!items.empty()) continue;  // the next tick
                    want = 1;                      // a lone pixel-heavy request still advances
                }
                if (q->r.slice_spp) want = std::min<uint64_t>(want, q->r.slice_spp);
                const uint32_t slice = (uint32_t)std::min<uint64_t>(want, q->r.spp - q->issued);
                budget -= std::min<uint64_t>(budget, (uint64_t)slice * px);
                items.push_back(grh::BatchItem{
                    gr_batch_item{q->r.scene_id, (float *)q->film.ptr, q->r.sample_offset + q->issued, slice},
                    (float *)q->comp.ptr, 1u});
                slices.emplace_back(id, slice);
                q->issued += slice;
                q->in_flight += slice;
            }
            if (items.empty()) {
                if (flight.empty()) {
                    if (sv->stop) break;
                    sv->cv_work.wait_for(lk, std::chrono::milliseconds(20));
                    continue;
                }
                // nothing new to issue: sleep until the oldest tick ends or a request
                // arrives (polling the event keeps arrivals from waiting on the tick)
                if (cudaEventQuery(flight.front().ev) == cudaErrorNotReady)
                    sv->cv_work.wait_for(lk, std::chrono::microseconds(200));
                continue;
            }
        }
        // 5. launch the tick
        if (!items.empty()) {
            Tick t;
            t.slices = slices;
            if (!spare.empty()) {
                t.ev = spare.back();
                spare.pop_back();
            } else if (cudaEventCreateWithFlags(&t.ev, cudaEventDisableTiming) != cudaSuccess) {
                t.ev = nullptr;
            }
            gr_status st;
            {
                std::lock_guard<std::mutex> lk(ctx->mu);
                st = grh::batch_enqueue(ctx, items.data(), (uint32_t)items.size(), 0u, ctx->stream);
                if (st == GR_OK && t.ev && cudaEventRecord(t.ev, ctx->stream) != cudaSuccess) st = GR_ECUDA;
                if (st == GR_OK && !t.ev) st = GR_ECUDA;
            }
            if (st != GR_OK) {
                // the whole tick failed: fail its requests (they may have partial films)
                cudaStreamSynchronize(ctx->stream);
                std::lock_guard<std::mutex> lk(sv->mu);
                for (auto &s : slices) {
                    Request *q = sv->reqs[s.first];
                    q->in_flight -= s.second;
                    q->cancel = true;
                    q->error = st;
                }
                if (t.ev) spare.push_back(t.ev);
                for (auto &s : slices) {
                    Request *q = sv->reqs[s.first];
                    std::vector<uint64_t> keep;
                    for (uint64_t id : sv->running)
                        if (id != q->id) keep.push_back(id);
                    sv->running.swap(keep);
                    finish(*sv, q, GR_REQ_FAILED, st);
                }
            } else {
                flight.push_back(std::move(t));
            }
        }
    }
    for (Tick &t : flight) cudaEventSynchronize(t.ev), spare.push_back(t.ev);
    for (cudaEvent_t e : spare)
        if (e) cudaEventDestroy(e);
}

// Metric sweeps, one at a time in arrival order (no context lock: own stream).  Each
// sweep's scratch is taken from the serve pool on the metrics stream and given back
// there: a growing cudaMalloc'd scratch would cudaFree the old one, which waits for
// the whole device -- measured on B200 to hold up the ticks and admissions for
// 0.1-0.9 s while a stone with more planes than any before was swept.
void metrics_main(gr_ctx *ctx, ServeState *sv) {
    cudaSetDevice(ctx->device);
    for (;;) {
        Request *q;
        {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv_metrics.wait(lk, [&] { return sv->stop || !sv->metric_queue.empty(); });
            if (sv->metric_queue.empty()) return;  // stopping, nothing left
            q = sv->reqs[sv->metric_queue.front()];
            sv->metric_queue.pop_front();
            if (q->cancel) {
                finish(*sv, q, GR_REQ_CANCELLED);
                continue;
            }
        }
        const uint32_t n_planes = (uint32_t)q->planes.size(), n_poses = (uint32_t)q->poses.size();
        grh::DeviceBuffer scratch;  // borrowed from the pool, never reserve-grown
        scratch.cap = grh::metrics_scratch_bytes(n_planes, n_poses);
        cudaError_t e = sv->film_pool ? cudaMallocFromPoolAsync(&scratch.ptr, scratch.cap, sv->film_pool, sv->metrics_stream)
                                      : cudaMallocAsync(&scratch.ptr, scratch.cap, sv->metrics_stream);
        gr_status st = GR_ENOMEM;
        if (e == cudaSuccess) {
            st = grh::metrics_device(q->planes.data(), n_planes, &q->material, q->poses.data(), n_poses,
                                     q->metrics.data(), q->r.flags, sv->metrics_stream, scratch);
            cudaFreeAsync(scratch.ptr, sv->metrics_stream);
        } else {
            cudaGetLastError();
        }
        std::lock_guard<std::mutex> lk(sv->mu);
        finish(*sv, q, st == GR_OK ? GR_REQ_DONE : GR_REQ_FAILED, st);
    }
}

ServeState *serve_state(gr_ctx *ctx) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (!ctx->serve) {
        ctx->serve = new ServeState();
        cudaSetDevice(ctx->device);
        int lo = 0, hi = 0;  // the numerically lowest priority is the highest
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        cudaStreamCreateWithPriority(&ctx->serve->metrics_stream, cudaStreamNonBlocking, hi);
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
            uint64_t keep = ctx->serve_budget;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            void *p = nullptr;
            if (cudaMallocFromPoolAsync(&p, std::min<uint64_t>(kFilmPoolReserve, ctx->serve_budget), pool,
                                        ctx->stream) == cudaSuccess)
                cudaFreeAsync(p, ctx->stream);  // mapped now, kept by the pool
            ctx->serve->film_pool = pool;
        }
        cudaGetLastError();  // a pool that could not be set up leaves films on the default pool
        // Scratch of a full tick and of each lane's full chunk, reserved now: growing a
        // buffer later frees the old one, which waits for the whole device (every
        // stream's work) and stalls the lanes behind it.
        ctx->xyz.reserve(std::max<size_t>(ctx->xyz.cap, 2 * kTickTuples * 3 * sizeof(float)));
        ctx->batch_tables.reserve(std::max<size_t>(ctx->batch_tables.cap, (size_t)1 << 20));
        ctx->batch_park.reserve(std::max<size_t>(ctx->batch_park.cap, 4096 + (kTickTuples / 16 + 32 * 1024) * sizeof(grd::Path)));
        // render lanes, their priorities below the metric sweeps' (the highest): by
        // default the smallest class next, the largest last
        for (int c = 0; c < kLaneClasses; ++c) {
            const int rank = GR_SERVE_LANE_ORDER ? kLaneClasses - 1 - c : c;
            const uint32_t n_lanes = GR_SERVE_POLICY == 1 ? (c == 2 ? GR_SERVE_CHUNK_LANES : 0) : kLanesPerClass[c];
            for (uint32_t k = 0; k < n_lanes; ++k) {
                // numerically larger = lower priority
                const int prio = std::min(lo, hi + 1 + (GR_SERVE_POLICY == 0 ? rank : 0));
                auto *L = new ServeState::Lane();
                L->cls = c;
                if (cudaStreamCreateWithPriority(&L->stream, cudaStreamNonBlocking, prio) != cudaSuccess) {
                    delete L;
                    continue;
                }
                L->xyz.reserve((size_t)kClassTuples[c] * 12);
                L->park.reserve(grh::staged_park_bytes(kClassTuples[c]));
                ctx->serve->lanes.push_back(L);
            }
        }
        cudaGetLastError();  // a reservation that failed is retried (grown) where it is used
        ctx->serve->worker = std::thread(worker_main, ctx, ctx->serve);
        ctx->serve->metrics_worker = std::thread(metrics_main, ctx, ctx->serve);
        for (auto *L : ctx->serve->lanes) L->th = std::thread(lane_main, ctx, ctx->serve, L);
    }
    return ctx->serve;
}

Request *find(ServeState *sv, uint64_t id) {
    auto it = sv->reqs.find(id);
    return it == sv->reqs.end() ? nullptr : it->second;
}

void fill_status(const Request *q, gr_request_status *out) {
    out->state = q->state;
    out->samples_done = q->done;
    out->error = q->error;
    out->queued_ms = q->state == GR_REQ_QUEUED ? ms_between(q->t_submit, Clock::now()) : ms_between(q->t_submit, q->t_admit);
    const bool ended = q->state == GR_REQ_DONE || q->state == GR_REQ_CANCELLED || q->state == GR_REQ_FAILED;
    out->latency_ms = ended ? ms_between(q->t_submit, q->t_done) : 0.0;
}

}  // namespace

namespace grh {
void serve_shutdown(gr_ctx *ctx) {
    ServeState *sv = ctx->serve;
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        for (auto &kv : sv->reqs) kv.second->cancel = true;
    }
    sv->cv_work.notify_all();
    sv->cv_metrics.notify_all();
    sv->cv_lane.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    if (sv->metrics_worker.joinable()) sv->metrics_worker.join();
    for (auto *L : sv->lanes)
        if (L->th.joinable()) L->th.join();
    cudaSetDevice(ctx->device);
    for (auto &kv : sv->reqs) {
        kv.second->film.release(ctx->stream);
        kv.second->comp.release(ctx->stream);
        if (kv.second->film_ev) cudaEventDestroy(kv.second->film_ev);
        delete kv.second;
    }
    cudaStreamSynchronize(ctx->stream);  // stream-ordered frees above complete
    if (sv->film_pool) cudaMemPoolDestroy(sv->film_pool);
    if (sv->metrics_stream) cudaStreamDestroy(sv->metrics_stream);
    for (auto *L : sv->lanes) {
        cudaStreamSynchronize(L->stream);
        cudaStreamDestroy(L->stream);
        L->xyz.release();
        L->park.release();
        delete L;
    }
    sv->lanes.clear();
    delete sv;
    ctx->serve = nullptr;
}
}  // namespace grh

extern "C" {

gr_status gr_submit(gr_ctx *ctx, const gr_request *req, uint64_t *request_id) {
    if (!ctx || !req || !request_id) return fail(GR_EINVAL, "NULL argument");
    const Clock::time_point t_entry = Clock::now();  // latency counts any wait for the locks below
    Request *q = new Request();
    q->r = *req;
    if (req->kind == GR_REQ_RENDER) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->scenes.find(req->scene_id);
        if (it == ctx->scenes.end()) {
            delete q;
            return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)req->scene_id);
        }
        q->n_px = (uint64_t)it->second->S.width * it->second->S.height;
        q->kahan = (it->second->S.flags & GR_FLAG_KAHAN_FILM) != 0;
        q->film_bytes = q->n_px * 3 * sizeof(float) * (q->kahan ? 2 : 1);
    } else if (req->kind == GR_REQ_METRICS) {
        if (!req->material || !req->poses || (req->n_planes && !req->planes) || req->n_planes > GR_MAX_PLANES) {
            delete q;
            return fail(GR_EINVAL, "metrics request needs material, poses and at most GR_MAX_PLANES planes");
        }
        q->poses.assign(req->poses, req->poses + req->n_poses);
        q->planes.assign(req->planes, req->planes + req->n_planes);
        q->material = *req->material;
        q->metrics.resize(req->n_poses);
        q->r.poses = nullptr;
        q->r.planes = nullptr;
        q->r.material = nullptr;
    } else {
        delete q;
        return fail(GR_EINVAL, "unknown request kind %u", req->kind);
    }
    ServeState *sv = serve_state(ctx);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        q->id = sv->next_id++;
        q->t_submit = t_entry;
        if (q->r.kind == GR_REQ_METRICS && q->r.n_planes == 0) {
            for (auto &m : q->metrics) m = gr_metrics_out{85.0f, 25.0f, 75.0f, 5.0f, 5.0f};  // color/metrics.rs:1090-1103
            q->t_admit = q->t_submit;
            finish(*sv, q, GR_REQ_DONE);
        } else if (q->r.kind == GR_REQ_RENDER && q->r.spp == 0) {
            q->t_admit = q->t_submit;
            finish(*sv, q, GR_REQ_DONE);
        } else if (q->r.kind == GR_REQ_METRICS) {
            q->state = GR_REQ_RUNNING;
            q->t_admit = q->t_submit;
            sv->metric_queue.push_back(q->id);
        } else {
            sv->queue.push_back(q->id);
        }
        sv->reqs[q->id] = q;
        *request_id = q->id;
        if (q->r.kind == GR_REQ_RENDER && q->state == GR_REQ_QUEUED) {
            // admitted here when its film fits, so a lane render starts without waiting
            // for a turn of the worker thread (which admits whatever stays queued)
            cudaSetDevice(ctx->device);
            admit(ctx, *sv, ctx->resident_bytes);
        }
    }
    if (q->r.kind == GR_REQ_METRICS)
        sv->cv_metrics.notify_all();
    else
        sv->cv_work.notify_all();
    return GR_OK;
}

gr_status gr_poll(gr_ctx *ctx, uint64_t id, gr_request_status *out) {
    if (!ctx || !out) return fail(GR_EINVAL, "NULL argument");
    if (!ctx->serve) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    ServeState *sv = ctx->serve;
    std::lock_guard<std::mutex> lk(sv->mu);
    Request *q = find(sv, id);
    if (!q) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    fill_status(q, out);
    return GR_OK;
}

gr_status gr_wait(gr_ctx *ctx, uint64_t id, uint32_t timeout_ms, gr_request_status *out) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (!ctx->serve) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    ServeState *sv = ctx->serve;
    std::unique_lock<std::mutex> lk(sv->mu);
    Request *q = find(sv, id);
    if (!q) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    auto ended = [&] { return q->state == GR_REQ_DONE || q->state == GR_REQ_CANCELLED || q->state == GR_REQ_FAILED; };
    if (!sv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ended)) {
        if (out) fill_status(q, out);
        return fail(GR_ETIMEOUT, "request %llu not finished after %u ms", (unsigned long long)id, timeout_ms);
    }
    if (out) fill_status(q, out);
    return GR_OK;
}

gr_status gr_cancel(gr_ctx *ctx, uint64_t id) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (!ctx->serve) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    ServeState *sv = ctx->serve;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        Request *q = find(sv, id);
        if (!q) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
        q->cancel = true;
    }
    sv->cv_work.notify_all();
    sv->cv_lane.notify_all();  // a lane render cancelled before its first chunk ends there
    return GR_OK;
}

gr_status gr_request_film(gr_ctx *ctx, uint64_t id, float *xyz_host) {
    if (!ctx || !xyz_host) return fail(GR_EINVAL, "NULL argument");
    if (!ctx->serve) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    ServeState *sv = ctx->serve;
    void *src = nullptr;
    uint64_t bytes = 0;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        Request *q = find(sv, id);
        if (!q) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
        if (q->r.kind != GR_REQ_RENDER) return fail(GR_EINVAL, "request %llu is not a render", (unsigned long long)id);
        if (q->state != GR_REQ_DONE && q->state != GR_REQ_CANCELLED)
            return fail(GR_EINVAL, "request %llu has not finished", (unsigned long long)id);
        src = q->film.ptr;
        bytes = q->n_px * 3 * sizeof(float);
    }
    if (!src) {
        std::memset(xyz_host, 0, bytes);  // finished before admission: no samples
        return GR_OK;
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    GR_CUDA(cudaSetDevice(ctx->device));
    GR_CUDA(cudaMemcpyAsync(xyz_host, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    GR_CUDA(cudaStreamSynchronize(ctx->stream));
    return GR_OK;
}

gr_status gr_request_metrics(gr_ctx *ctx, uint64_t id, gr_metrics_out *out) {
    if (!ctx || !out) return fail(GR_EINVAL, "NULL argument");
    if (!ctx->serve) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    ServeState *sv = ctx->serve;
    std::lock_guard<std::mutex> lk(sv->mu);
    Request *q = find(sv, id);
    if (!q) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    if (q->r.kind != GR_REQ_METRICS || q->state != GR_REQ_DONE)
        return fail(GR_EINVAL, "request %llu is not a finished metrics request", (unsigned long long)id);
    for (size_t i = 0; i < q->metrics.size(); ++i) out[i] = q->metrics[i];
    return GR_OK;
}

gr_status gr_request_release(gr_ctx *ctx, uint64_t id) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    if (!ctx->serve) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
    ServeState *sv = ctx->serve;
    Request *q = nullptr;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        q = find(sv, id);
        if (!q) return fail(GR_ENOTFOUND, "unknown request id %llu", (unsigned long long)id);
        if (q->state == GR_REQ_QUEUED || q->state == GR_REQ_RUNNING)
            return fail(GR_EBUSY, "request %llu is still active (cancel it first)", (unsigned long long)id);
        if (q->admitted) sv->film_bytes -= q->film_bytes;
        sv->reqs.erase(id);
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    q->film.release(ctx->stream);  // stream-ordered: after every tick that wrote it
    q->comp.release(ctx->stream);
    if (q->film_ev) cudaEventDestroy(q->film_ev);
    delete q;
    return GR_OK;
}

}  // extern "C"
