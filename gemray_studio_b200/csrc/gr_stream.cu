// gr_stream.cu -- frame-delta streaming of one render request: gr_stream_*.
//
// The worker's stream emitter (apps/gemray-worker/src/stream_emit/) splits a render
// into a free-running tracer and an emitter that drains on the client's cadence; the
// two meet only at a mutex-protected pending delta and running total.  Here the tracer
// is a host thread per stream that issues the sub-batches on the stream's own CUDA
// stream (`main`), and the drains run on a second CUDA stream (`side`):
//
//   tracer, per sub-batch:  zero `batch`; trace + fold the sub-batch into it (the film
//       one trace_samples_with_gpu call returns) and wait for it; then, under the
//       stream mutex, wait for the side stream's last drain, fold `batch` into
//       pending[cur] (copy when that buffer is empty, else add) and into `total`
//       (add), record `folded`.
//   drain (gr_stream_take): under the mutex, swap cur to the other pending buffer
//       (which starts empty), make the side stream wait for `folded`, copy the old
//       buffer to the host there and record `drained`.  The next fold waits for
//       `drained`, so a buffer is never refilled while it is being copied, and a drain
//       never waits for the sub-batch being traced.
//   total / preview: the same pattern on `total`, no swap.
//
// Arithmetic: every sub-batch sum starts from a zero film and pending / total add
// them in sub-batch order with plain f32 adds -- PendingDelta::add and the
// `running_total += buf` loop (tracer.rs:93-100) -- so a run with a given sub-batch
// split reproduces the reference's values for that split.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>

#include "gr_ctx.h"
#include "gr_launch.cuh"

using grh::fail;

namespace grd {

// pending = copy ? batch : pending + batch; total += batch (elementwise over W*H*3)
__global__ void k_stream_fold(const float *__restrict__ batch, float *__restrict__ pending, float *__restrict__ total,
                              uint64_t n, uint32_t copy) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float b = batch[i];
        pending[i] = copy ? b : pending[i] + b;
        total[i] = total[i] + b;
    }
}

// downsample_preview (stream_emit/downsample.rs:17-53): output pixel (ox, oy) is the
// mean of source rows [oy*h/th, max((oy+1)*h/th, y0+1) min h) x the same for columns,
// summed row by row from zero, divided by the count as f32.
__global__ void k_downsample_preview(const float *__restrict__ src, uint32_t w, uint32_t h, uint32_t tw, uint32_t th,
                                     float *__restrict__ out) {
    const uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= (uint64_t)tw * th) return;
    const uint64_t oy = o / tw, ox = o % tw;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    uint32_t count = 0;
    if (w != 0 && h != 0) {
        const uint64_t y0 = oy * h / th;
        uint64_t y1 = (oy + 1) * h / th;
        if (y1 < y0 + 1) y1 = y0 + 1;
        if (y1 > h) y1 = h;
        const uint64_t x0 = ox * w / tw;
        uint64_t x1 = (ox + 1) * w / tw;
        if (x1 < x0 + 1) x1 = x0 + 1;
        if (x1 > w) x1 = w;
        for (uint64_t y = y0; y < y1; ++y) {
            const float *row = src + 3 * (y * w);
            for (uint64_t x = x0; x < x1; ++x) {
                sx = sx + row[3 * x + 0];
                sy = sy + row[3 * x + 1];
                sz = sz + row[3 * x + 2];
                ++count;
            }
        }
    }
    if (count == 0) {
        sx = sy = sz = 0.0f;
    } else {
        const float c = (float)count;
        sx = sx / c;
        sy = sy / c;
        sz = sz / c;
    }
    out[3 * o + 0] = sx;
    out[3 * o + 1] = sy;
    out[3 * o + 2] = sz;
}

}  // namespace grd

struct FrameStream {
    gr_ctx *ctx = nullptr;
    ResidentScene *rs = nullptr;
    SceneConst S;
    grd::SceneBuffers B;
    StageCaps caps;  // the scene's stage caps as chosen when the stream opened
    uint32_t first = 0, samples = 0;
    double target_ms = 100.0;
    uint32_t first_batch = 1, fixed_batch = 0;
    uint64_t n_pixels = 0;
    cudaStream_t main = nullptr, side = nullptr;
    cudaEvent_t folded = nullptr, drained = nullptr, t0 = nullptr, t1 = nullptr;
    bool drained_recorded = false;
    grh::DeviceBuffer scratch, batch, pending[2], total, preview, park;
    std::mutex mu;       // tracer <-> drains: cur, empty, range, progress, state
    std::mutex emit_mu;  // serialises the drains (take / total / preview) of this stream
    int cur = 0;
    bool empty[2] = {true, true};
    uint32_t range_first = 0, range_samples = 0;
    uint32_t samples_done = 0;
    uint32_t state = GR_STREAM_RUNNING;
    gr_status error = GR_OK;
    std::string error_msg;  // the tracer thread's message (error strings are per thread)
    bool discarded = false;  // cancelled: pending deltas are dropped, not drained
    std::atomic<bool> cancel{false};
    std::thread tracer;
};

namespace {

constexpr size_t kStreamScratchBudget = 256ull << 20;  // per-stream XYZ scratch per launch

gr_status stream_fail(FrameStream *fs, gr_status st) {
    std::lock_guard<std::mutex> lk(fs->mu);
    fs->error = st;
    fs->error_msg = gr_last_error_string();
    fs->state = GR_STREAM_FAILED;
    return st;
}

// One sub-batch [bfirst, bfirst + n) traced into fs->batch (zeroed first), in chunks
// of whole pixels through the stream's own scratch on its own CUDA stream.
gr_status trace_subbatch(FrameStream *fs, uint32_t bfirst, uint32_t n) {
    const size_t film_bytes = (size_t)fs->n_pixels * 3 * sizeof(float);
    GR_CUDA(cudaMemsetAsync(fs->batch.ptr, 0, film_bytes, fs->main));
    uint64_t chunk_pixels = (kStreamScratchBudget / (3 * sizeof(float))) / n;
    if (chunk_pixels < 1) chunk_pixels = 1;
    if (chunk_pixels > fs->n_pixels) chunk_pixels = fs->n_pixels;
    gr_status st = fs->scratch.reserve((size_t)chunk_pixels * n * 3 * sizeof(float));
    if (st != GR_OK) return st;
    for (uint64_t p0 = 0; p0 < fs->n_pixels; p0 += chunk_pixels) {
        const uint64_t np = fs->n_pixels - p0 < chunk_pixels ? fs->n_pixels - p0 : chunk_pixels;
        grd::LaunchRange R;
        R.first_pixel = (uint32_t)p0;
        R.n_pixels = (uint32_t)np;
        R.sample_offset = bfirst;
        R.spp = n;
        R.n_tuples = np * n;
        st = grh::launch_trace(fs->ctx, fs->S, fs->B, R, (float *)fs->scratch.ptr, fs->main, GR_KERNEL_AUTO,
                               &fs->park, fs->caps);
        if (st != GR_OK) return st;
        st = grh::launch_fold((const float *)fs->scratch.ptr, (uint32_t)np, n, (uint32_t)p0, (float *)fs->batch.ptr,
                              (fs->S.flags & GR_FLAG_KAHAN_FILM) ? 1u : 0u, fs->main);
        if (st != GR_OK) return st;
    }
    return GR_OK;
}

// run_tracer (stream_emit/tracer.rs:64-117) on the stream's CUDA stream.
void tracer_main(FrameStream *fs) {
    if (cudaSetDevice(fs->ctx->device) != cudaSuccess) {
        stream_fail(fs, fail(GR_ECUDA, "cudaSetDevice failed in the stream tracer"));
        return;
    }
    const uint64_t n3 = fs->n_pixels * 3;
    const unsigned threads = 256;
    uint64_t blocks = (n3 + threads - 1) / threads;
    const uint64_t max_blocks = (uint64_t)(fs->ctx->sm_count > 0 ? fs->ctx->sm_count : 148) * 8;
    if (blocks > max_blocks) blocks = max_blocks;
    if (blocks == 0) blocks = 1;
    uint32_t produced = 0;
    uint32_t batch_size = fs->fixed_batch ? fs->fixed_batch : (fs->first_batch ? fs->first_batch : 1);
    while (produced < fs->samples) {
        if (fs->cancel.load(std::memory_order_relaxed)) break;
        const uint32_t left = fs->samples - produced;
        const uint32_t this_batch = batch_size < left ? batch_size : left;
        const uint32_t bfirst = fs->first + produced;
        gr_status st = GR_OK;
        if (cudaEventRecord(fs->t0, fs->main) != cudaSuccess) st = fail(GR_ECUDA, "cudaEventRecord failed");
        if (st == GR_OK) st = trace_subbatch(fs, bfirst, this_batch);
        if (st == GR_OK && cudaEventRecord(fs->t1, fs->main) != cudaSuccess) st = fail(GR_ECUDA, "cudaEventRecord failed");
        // The fold is enqueued only once the sub-batch has been traced, so the `folded`
        // event a drain waits for is never queued behind a sub-batch in progress.
        float ms = 0.0f;
        if (st == GR_OK) {
            cudaError_t e = cudaEventSynchronize(fs->t1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, fs->t0, fs->t1);
            if (e != cudaSuccess) st = fail(GR_ECUDA, "sub-batch failed: %s", cudaGetErrorString(e));
        }
        if (st != GR_OK) {
            stream_fail(fs, st);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(fs->mu);
            cudaError_t e = cudaSuccess;
            if (fs->drained_recorded) e = cudaStreamWaitEvent(fs->main, fs->drained, 0);
            const int c = fs->cur;
            if (e == cudaSuccess) {
                grd::k_stream_fold<<<(unsigned)blocks, threads, 0, fs->main>>>(
                    (const float *)fs->batch.ptr, (float *)fs->pending[c].ptr, (float *)fs->total.ptr, n3,
                    fs->empty[c] ? 1u : 0u);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaEventRecord(fs->folded, fs->main);
            if (e != cudaSuccess) {
                fs->error = fail(GR_ECUDA, "stream fold failed: %s", cudaGetErrorString(e));
                fs->error_msg = gr_last_error_string();
                fs->state = GR_STREAM_FAILED;
                return;
            }
            if (fs->empty[c]) {
                fs->empty[c] = false;
                fs->range_first = bfirst;
                fs->range_samples = this_batch;
            } else {
                fs->range_samples += this_batch;  // sub-batches arrive in contiguous order
            }
            produced += this_batch;
            fs->samples_done = produced;
        }
        if (!fs->fixed_batch) batch_size = gr_next_batch_size(batch_size, (double)ms, fs->target_ms);
    }
    // the last fold must be complete before the stream reports it
    cudaError_t e = cudaEventSynchronize(fs->folded);
    std::lock_guard<std::mutex> lk(fs->mu);
    if (e != cudaSuccess) {
        fs->error = fail(GR_ECUDA, "stream fold failed: %s", cudaGetErrorString(e));
        fs->error_msg = gr_last_error_string();
        fs->state = GR_STREAM_FAILED;
    } else {
        fs->state = produced < fs->samples ? GR_STREAM_CANCELLED : GR_STREAM_FINISHED;
    }
}

FrameStream *find_stream(gr_ctx *ctx, uint64_t id) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->streams.find(id);
    return it == ctx->streams.end() ? nullptr : it->second;
}

// Copies `src` (device, W*H*3 floats unless n3 given) to the host on the side stream
// after the last fold; the caller holds fs->emit_mu and fs->mu.
gr_status side_copy_locked(FrameStream *fs, const void *src, size_t bytes, float *host) {
    GR_CUDA(cudaStreamWaitEvent(fs->side, fs->folded, 0));
    GR_CUDA(cudaMemcpyAsync(host, src, bytes, cudaMemcpyDeviceToHost, fs->side));
    GR_CUDA(cudaEventRecord(fs->drained, fs->side));
    fs->drained_recorded = true;
    return GR_OK;
}

void destroy_stream(FrameStream *fs) {
    fs->cancel.store(true);
    if (fs->tracer.joinable()) fs->tracer.join();
    cudaSetDevice(fs->ctx->device);
    if (fs->main) cudaStreamSynchronize(fs->main);
    if (fs->side) cudaStreamSynchronize(fs->side);
    fs->scratch.release();
    fs->batch.release();
    fs->pending[0].release();
    fs->pending[1].release();
    fs->total.release();
    fs->preview.release();
    fs->park.release();
    for (cudaEvent_t ev : {fs->folded, fs->drained, fs->t0, fs->t1})
        if (ev) cudaEventDestroy(ev);
    if (fs->main) cudaStreamDestroy(fs->main);
    if (fs->side) cudaStreamDestroy(fs->side);
    delete fs;
}

}  // namespace

namespace grh {
void streams_shutdown(gr_ctx *ctx) {
    std::map<uint64_t, FrameStream *> all;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        all.swap(ctx->streams);
        for (auto &kv : all)
            if (kv.second->rs && kv.second->rs->users) kv.second->rs->users--;
    }
    for (auto &kv : all) destroy_stream(kv.second);
}
}  // namespace grh

extern "C" {

uint32_t gr_next_batch_size(uint32_t prev, double elapsed_ms, double target_ms) {
    const uint64_t grown = (uint64_t)prev * 4u;
    const uint32_t max_growth_u = grown > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)(grown ? grown : 1u);
    if (!(elapsed_ms > 0.0)) return max_growth_u;
    const double scaled = (double)prev * (target_ms / elapsed_ms);
    double v = scaled < 1.0 ? 1.0 : scaled;
    if (v > (double)max_growth_u) v = (double)max_growth_u;
    return (uint32_t)std::round(v);
}

gr_status gr_stream_open(gr_ctx *ctx, uint64_t scene_id, uint32_t first_sample, uint32_t samples,
                         const gr_stream_opts *opts, uint64_t *out_stream) {
    if (!ctx || !out_stream) return fail(GR_EINVAL, "ctx or out_stream is NULL");
    FrameStream *fs = new FrameStream();
    fs->ctx = ctx;
    fs->first = first_sample;
    fs->samples = samples;
    if (opts) {
        if (opts->target_ms) fs->target_ms = (double)opts->target_ms;
        if (opts->first_batch) fs->first_batch = opts->first_batch;
        fs->fixed_batch = opts->fixed_batch;
    }
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->scenes.find(scene_id);
        if (it == ctx->scenes.end()) {
            delete fs;
            return fail(GR_ENOTFOUND, "unknown scene id %llu", (unsigned long long)scene_id);
        }
        fs->rs = it->second;
        fs->S = fs->rs->S;
        fs->B = resident_buffers(fs->rs);
        fs->caps = grh::scene_stage_caps(*fs->rs);
        fs->rs->users++;
    }
    fs->n_pixels = (uint64_t)fs->S.width * fs->S.height;
    auto undo = [&](gr_status st) {
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            fs->rs->users--;
        }
        destroy_stream(fs);
        return st;
    };
    if (cudaSetDevice(ctx->device) != cudaSuccess) return undo(fail(GR_ECUDA, "cudaSetDevice failed"));
    const size_t film_bytes = (size_t)(fs->n_pixels ? fs->n_pixels : 1) * 3 * sizeof(float);
    if (cudaStreamCreateWithFlags(&fs->main, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&fs->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&fs->folded, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&fs->drained, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&fs->t0) != cudaSuccess || cudaEventCreate(&fs->t1) != cudaSuccess)
        return undo(fail(GR_ECUDA, "stream / event creation failed"));
    gr_status st = fs->batch.reserve(film_bytes);
    if (st == GR_OK) st = fs->pending[0].reserve(film_bytes);
    if (st == GR_OK) st = fs->pending[1].reserve(film_bytes);
    if (st == GR_OK) st = fs->total.reserve(film_bytes);
    if (st != GR_OK) return undo(st);
    if (cudaMemsetAsync(fs->total.ptr, 0, film_bytes, fs->main) != cudaSuccess ||
        cudaEventRecord(fs->folded, fs->main) != cudaSuccess)
        return undo(fail(GR_ECUDA, "stream initialisation failed"));
    if (fs->n_pixels == 0 || samples == 0) {
        fs->state = GR_STREAM_FINISHED;
    } else {
        try {
            fs->tracer = std::thread(tracer_main, fs);
        } catch (...) {
            return undo(fail(GR_ENOMEM, "could not start the stream tracer thread"));
        }
    }
    std::lock_guard<std::mutex> lk(ctx->mu);
    const uint64_t id = ctx->next_stream_id++;
    ctx->streams[id] = fs;
    *out_stream = id;
    return GR_OK;
}

gr_status gr_stream_take(gr_ctx *ctx, uint64_t stream, uint32_t *first_sample, uint32_t *samples, float *xyz_host) {
    if (!ctx || !first_sample || !samples) return fail(GR_EINVAL, "NULL argument");
    FrameStream *fs = find_stream(ctx, stream);
    if (!fs) return fail(GR_ENOTFOUND, "unknown stream id %llu", (unsigned long long)stream);
    std::lock_guard<std::mutex> elk(fs->emit_mu);
    *first_sample = 0;
    *samples = 0;
    {
        std::lock_guard<std::mutex> lk(fs->mu);
        const int c = fs->cur;
        if (fs->discarded || fs->empty[c]) return GR_OK;
        if (!xyz_host) return fail(GR_EINVAL, "xyz_host is NULL");
        GR_CUDA(cudaSetDevice(ctx->device));
        gr_status st = side_copy_locked(fs, fs->pending[c].ptr, (size_t)fs->n_pixels * 3 * sizeof(float), xyz_host);
        if (st != GR_OK) return st;
        *first_sample = fs->range_first;
        *samples = fs->range_samples;
        fs->cur = c ^ 1;
        fs->empty[c ^ 1] = true;
    }
    GR_CUDA(cudaEventSynchronize(fs->drained));
    return GR_OK;
}

gr_status gr_stream_status(gr_ctx *ctx, uint64_t stream, uint32_t *samples_done, uint32_t *state,
                           gr_status *tracer_error) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    FrameStream *fs = find_stream(ctx, stream);
    if (!fs) return fail(GR_ENOTFOUND, "unknown stream id %llu", (unsigned long long)stream);
    std::lock_guard<std::mutex> lk(fs->mu);
    if (samples_done) *samples_done = fs->samples_done;
    if (state) *state = fs->state;
    if (tracer_error) *tracer_error = fs->error;
    // make the tracer's message readable from this thread's gr_last_error_string()
    if (fs->state == GR_STREAM_FAILED) fail(fs->error, "stream tracer: %s", fs->error_msg.c_str());
    return GR_OK;
}

gr_status gr_stream_total(gr_ctx *ctx, uint64_t stream, float *xyz_host) {
    if (!ctx || !xyz_host) return fail(GR_EINVAL, "NULL argument");
    FrameStream *fs = find_stream(ctx, stream);
    if (!fs) return fail(GR_ENOTFOUND, "unknown stream id %llu", (unsigned long long)stream);
    std::lock_guard<std::mutex> elk(fs->emit_mu);
    {
        std::lock_guard<std::mutex> lk(fs->mu);
        GR_CUDA(cudaSetDevice(ctx->device));
        gr_status st = side_copy_locked(fs, fs->total.ptr, (size_t)fs->n_pixels * 3 * sizeof(float), xyz_host);
        if (st != GR_OK) return st;
    }
    GR_CUDA(cudaEventSynchronize(fs->drained));
    return GR_OK;
}

gr_status gr_stream_preview(gr_ctx *ctx, uint64_t stream, uint32_t tw, uint32_t th, float *xyz_host) {
    if (!ctx || !xyz_host) return fail(GR_EINVAL, "NULL argument");
    FrameStream *fs = find_stream(ctx, stream);
    if (!fs) return fail(GR_ENOTFOUND, "unknown stream id %llu", (unsigned long long)stream);
    if (tw == 0) tw = 1;
    if (th == 0) th = 1;
    const uint64_t n_out = (uint64_t)tw * th;
    if (n_out > (1ull << 28)) return fail(GR_EINVAL, "preview %ux%u is too large", tw, th);
    std::lock_guard<std::mutex> elk(fs->emit_mu);
    {
        std::lock_guard<std::mutex> lk(fs->mu);
        GR_CUDA(cudaSetDevice(ctx->device));
        gr_status st = fs->preview.reserve((size_t)n_out * 3 * sizeof(float));
        if (st != GR_OK) return st;
        GR_CUDA(cudaStreamWaitEvent(fs->side, fs->folded, 0));
        const unsigned threads = 128;
        grd::k_downsample_preview<<<(unsigned)((n_out + threads - 1) / threads), threads, 0, fs->side>>>(
            (const float *)fs->total.ptr, fs->S.width, fs->S.height, tw, th, (float *)fs->preview.ptr);
        GR_CUDA(cudaGetLastError());
        GR_CUDA(cudaMemcpyAsync(xyz_host, fs->preview.ptr, (size_t)n_out * 3 * sizeof(float), cudaMemcpyDeviceToHost,
                                fs->side));
        GR_CUDA(cudaEventRecord(fs->drained, fs->side));
        fs->drained_recorded = true;
    }
    GR_CUDA(cudaEventSynchronize(fs->drained));
    return GR_OK;
}

gr_status gr_stream_cancel(gr_ctx *ctx, uint64_t stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    FrameStream *fs = find_stream(ctx, stream);
    if (!fs) return fail(GR_ENOTFOUND, "unknown stream id %llu", (unsigned long long)stream);
    fs->cancel.store(true);
    std::lock_guard<std::mutex> lk(fs->mu);
    fs->discarded = true;
    return GR_OK;
}

gr_status gr_stream_close(gr_ctx *ctx, uint64_t stream) {
    if (!ctx) return fail(GR_EINVAL, "ctx is NULL");
    FrameStream *fs = nullptr;
    {
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto it = ctx->streams.find(stream);
        if (it == ctx->streams.end()) return fail(GR_ENOTFOUND, "unknown stream id %llu", (unsigned long long)stream);
        fs = it->second;
        ctx->streams.erase(it);
        if (fs->rs && fs->rs->users) fs->rs->users--;
    }
    destroy_stream(fs);
    return GR_OK;
}

}  // extern "C"
