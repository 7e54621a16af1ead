// Asynchronous slot-pool uploads (streaming residency).
//
// addBatches (ComputeRasteriserPointCloud.swift:410-452) copies a chunk's
// points into free slots and marks them resident at once; the reference's
// StreamingAdapter (StreamingAdapter.swift:71-177) calls it from the render
// loop, so every upload is a main-thread copy that the frame waits for.  Here
// the copy is asynchronous:
//
//   * the caller's arrays are copied (host memcpy) into a page-locked staging
//     ring of the cloud and are free again when the call returns; or, with
//     CR_UPLOAD_BORROW, the caller's own page-locked arrays are the source of
//     the device copies and stay borrowed until the upload is published (no
//     host copy at all: a streaming source that keeps its chunks pinned);
//   * the staging bytes go to the slots' pool ranges on the context's upload
//     stream, after the render work enqueued before the call (a slot freed in
//     the same tick may still be read by an earlier frame);
//   * the slots leave the free list at once but stay non-resident (state 0,
//     which the cull skips) until the copy has landed: cr_cloud_poll_uploads
//     checks the copies' events without blocking and publishes the landed
//     slots as resident (state 1), so a frame never draws a half-copied slot;
//   * removing a slot whose copy is still in flight cancels it: the slot
//     returns to the free list when the copy lands.
//
// Uploads land in the order they were enqueued (one stream), so the staging
// ring is released from its tail.
#include <cstring>

#include "cr_internal.h"

using cri::fail;

namespace {

constexpr uint64_t kDefaultStaging = 64ull << 20;

uint64_t align16(uint64_t x) { return (x + 15) & ~uint64_t(15); }

// Staging bytes of n points: four 32-bit arrays and the level bytes, each
// 16-byte aligned.
uint64_t staging_bytes(uint64_t n) { return 4 * align16(4 * n) + align16(n); }

UploadState &state(cr_cloud *c) {
    if (!c->up) {
        c->up = new UploadState();
        c->up->slot.assign(c->cap.maxResidentBatches, 0);
    }
    return *c->up;
}

// Publishes the oldest upload, whose copies have completed.
void land_front(cr_cloud *c) {
    UploadState &u = *c->up;
    PendingUpload &p = u.q.front();
    for (const UploadBatch &b : p.batches) {
        if (u.slot[b.slot] == kSlotPending) {
            c->mirror[b.slot] = b.rec;
            mark_dirty(c, b.slot, b.slot);
            c->resident += 1;
            c->points += b.rec.numPoints;
        } else {  // removed while in flight
            c->free_slots.push_back(b.slot);
        }
        u.slot[b.slot] = kSlotIdle;
        u.in_flight_batches -= 1;
    }
    u.spare.push_back(p.ev);
    u.q.pop_front();
    if (u.q.empty())
        u.head = u.tail = 0;
    else
        u.tail = u.q.front().stage_off;
}

// Lands completed uploads from the front; with `block`, waits for all.
cr_status land(cr_cloud *c, bool block, uint32_t *landed) {
    if (!c->up) return CR_OK;
    UploadState &u = *c->up;
    while (!u.q.empty()) {
        cudaEvent_t ev = u.q.front().ev;
        if (block) {
            CR_CUDA(cudaEventSynchronize(ev));
        } else {
            const cudaError_t e = cudaEventQuery(ev);
            if (e == cudaErrorNotReady) break;
            if (e != cudaSuccess) return cri::cuda_fail(e, "cudaEventQuery");
        }
        if (landed) *landed += (uint32_t)u.q.front().batches.size();
        land_front(c);
    }
    return CR_OK;
}

// A staging region of `need` bytes (ring order), or -1 if the ring has no
// contiguous room now.
int64_t ring_alloc(UploadState &u, uint64_t need) {
    if (u.q.empty()) {
        u.head = u.tail = 0;
        return need <= u.cap ? 0 : -1;
    }
    if (u.head > u.tail) {
        if (u.cap - u.head >= need) return (int64_t)u.head;
        if (u.tail >= need) return 0;  // wrap
        return -1;
    }
    if (u.head < u.tail && u.tail - u.head >= need) return (int64_t)u.head;
    return -1;  // head == tail with uploads in flight: full
}

}  // namespace

cr_status uploads_drain(cr_cloud *c) {
    if (!c->up || c->up->q.empty()) return CR_OK;
    DeviceGuard g(c->ctx->device);
    return land(c, true, nullptr);
}

void uploads_free(cr_cloud *c) {
    if (!c->up) return;
    UploadState &u = *c->up;
    for (PendingUpload &p : u.q) {
        cudaEventSynchronize(p.ev);
        cudaEventDestroy(p.ev);
    }
    for (cudaEvent_t e : u.spare) cudaEventDestroy(e);
    if (u.ready) cudaEventDestroy(u.ready);
    if (u.h_stage) cudaFreeHost(u.h_stage);
    delete c->up;
    c->up = nullptr;
}

bool uploads_cancel(cr_cloud *c, int32_t slot) {
    if (!c->up || c->up->slot[slot] == kSlotIdle) return false;
    c->up->slot[slot] = kSlotCancelled;  // freed when its copy lands
    return true;
}

bool upload_slot_busy(const cr_cloud *c, uint32_t slot) {
    return c->up && c->up->slot[slot] != kSlotIdle;
}

extern "C" {

CR_API cr_status cr_cloud_add_batches_async(cr_cloud *c, const uint32_t *low, const uint32_t *med,
                                            const uint32_t *high, const uint32_t *colors,
                                            const uint8_t *levels, uint64_t points_len,
                                            const cr_raster_batch *batches, uint32_t n,
                                            uint32_t flags, int32_t *slots_out) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    if (n > c->free_slots.size())
        return fail(CR_ERR_CAPACITY, "addBatches: not enough free slots (have " +
                                         std::to_string(c->free_slots.size()) + ", need " +
                                         std::to_string(n) + ")");
    if (n == 0) return CR_OK;
    if (!batches || !low || !med || !high || !colors || !levels)
        return fail(CR_ERR_INVALID_ARGUMENT, "null array");
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t src = batches[i].firstPoint, cnt = batches[i].numPoints;
        if (cnt > c->cap.pointsPerBatch)
            return fail(CR_ERR_CAPACITY, "batch numPoints (" + std::to_string(cnt) +
                                             ") exceeds slot capacity (" +
                                             std::to_string(c->cap.pointsPerBatch) + ")");
        if (src + cnt > points_len)
            return fail(CR_ERR_INVALID_ARGUMENT, "addBatches: source data too small for batch");
        if (batches[i].fileIndex >= c->files.size())
            return fail(CR_ERR_INVALID_ARGUMENT, "batch fileIndex outside the file table");
        total += cnt;
    }
    if (flags & ~(uint32_t)CR_UPLOAD_BORROW)
        return fail(CR_ERR_INVALID_ARGUMENT, "unknown upload flags");
    const bool borrow = (flags & CR_UPLOAD_BORROW) != 0;
    cr_context *ctx = c->ctx;
    DeviceGuard g(ctx->device);
    UploadState &u = state(c);
    const uint64_t need = borrow ? 0 : staging_bytes(total);
    if (need > 0 && need > u.cap) {
        // Grow the ring (after every copy out of the old one has landed).
        cr_status st = land(c, true, nullptr);
        if (st) return st;
        if (u.h_stage) CR_CUDA(cudaFreeHost(u.h_stage));
        u.h_stage = nullptr;
        u.cap = 0;
        const uint64_t cap = std::max(need, u.want_cap ? u.want_cap : kDefaultStaging);
        CR_CUDA(cudaHostAlloc((void **)&u.h_stage, cap, cudaHostAllocDefault));
        u.cap = cap;
    }
    if (!ctx->upload_stream)
        CR_CUDA(cudaStreamCreateWithFlags(&ctx->upload_stream, cudaStreamNonBlocking));
    if (!u.ready) CR_CUDA(cudaEventCreateWithFlags(&u.ready, cudaEventDisableTiming));
    PendingUpload p;
    p.batches.reserve(n);
    // Source of the device copies: the caller's page-locked arrays (borrowed
    // until the upload is published), indexed by the batches' firstPoint; or
    // a staging region holding the batches' points back to back.
    const uint32_t *s_low = low, *s_med = med, *s_high = high, *s_col = colors;
    const uint8_t *s_lv = levels;
    if (borrow) {
        p.stage_off = u.head;  // holds no staging bytes
    } else {
        int64_t off;
        while ((off = ring_alloc(u, need)) < 0) {
            // No room: wait for the oldest upload to land.
            CR_CUDA(cudaEventSynchronize(u.q.front().ev));
            land_front(c);
        }
        u.head = (uint64_t)off + need;
        if (u.q.empty()) u.tail = (uint64_t)off;
        p.stage_off = (uint64_t)off;
        // Host copy into the staging region: the four word arrays and the
        // level bytes of all batches, batch after batch.
        unsigned char *base = u.h_stage + off;
        const uint64_t w4 = align16(4 * total);
        uint32_t *d_low = reinterpret_cast<uint32_t *>(base);
        uint32_t *d_med = reinterpret_cast<uint32_t *>(base + w4);
        uint32_t *d_high = reinterpret_cast<uint32_t *>(base + 2 * w4);
        uint32_t *d_col = reinterpret_cast<uint32_t *>(base + 3 * w4);
        uint8_t *d_lv = base + 4 * w4;
        uint64_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const uint64_t src = batches[i].firstPoint, cnt = batches[i].numPoints;
            std::memcpy(d_low + k, low + src, cnt * 4);
            std::memcpy(d_med + k, med + src, cnt * 4);
            std::memcpy(d_high + k, high + src, cnt * 4);
            std::memcpy(d_col + k, colors + src, cnt * 4);
            std::memcpy(d_lv + k, levels + src, cnt);
            k += cnt;
        }
        s_low = d_low;
        s_med = d_med;
        s_high = d_high;
        s_col = d_col;
        s_lv = d_lv;
    }

    // Device copies after the render work enqueued so far.
    cudaStream_t us = ctx->upload_stream;
    CR_CUDA(cudaEventRecord(u.ready, ctx->stream));
    CR_CUDA(cudaStreamWaitEvent(us, u.ready, 0));
    uint64_t run_src = 0, run_dst = 0, run_n = 0;
    auto flush_run = [&]() -> cr_status {
        if (run_n == 0) return CR_OK;
        CR_CUDA(cudaMemcpyAsync(c->d_low + run_dst, s_low + run_src, run_n * 4,
                                cudaMemcpyHostToDevice, us));
        CR_CUDA(cudaMemcpyAsync(c->d_med + run_dst, s_med + run_src, run_n * 4,
                                cudaMemcpyHostToDevice, us));
        CR_CUDA(cudaMemcpyAsync(c->d_high + run_dst, s_high + run_src, run_n * 4,
                                cudaMemcpyHostToDevice, us));
        CR_CUDA(cudaMemcpyAsync(c->d_colors + run_dst, s_col + run_src, run_n * 4,
                                cudaMemcpyHostToDevice, us));
        CR_CUDA(cudaMemcpyAsync(c->d_levels + run_dst, s_lv + run_src, run_n,
                                cudaMemcpyHostToDevice, us));
        run_n = 0;
        return CR_OK;
    };
    uint64_t k = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const int32_t slot = c->free_slots.back();
        c->free_slots.pop_back();
        if (slots_out) slots_out[i] = slot;
        const uint64_t dst = (uint64_t)slot * c->cap.pointsPerBatch;
        const uint64_t cnt = batches[i].numPoints;
        const uint64_t src = borrow ? (uint64_t)batches[i].firstPoint : k;
        if (cnt > 0) {
            if (run_n > 0 && run_src + run_n == src && run_dst + run_n == dst) {
                run_n += cnt;
            } else {
                cr_status st = flush_run();
                if (st) return st;
                run_src = src;
                run_dst = dst;
                run_n = cnt;
            }
        }
        k += cnt;
        UploadBatch b;
        b.slot = slot;
        b.rec = batches[i];
        b.rec.firstPoint = (uint32_t)dst;
        b.rec.state = 1;
        p.batches.push_back(b);
        u.slot[slot] = kSlotPending;
    }
    cr_status st = flush_run();
    if (st) return st;
    if (!u.spare.empty()) {
        p.ev = u.spare.back();
        u.spare.pop_back();
    } else {
        CR_CUDA(cudaEventCreateWithFlags(&p.ev, cudaEventDisableTiming));
    }
    CR_CUDA(cudaEventRecord(p.ev, us));
    u.in_flight_batches += n;
    u.q.push_back(std::move(p));
    return CR_OK;
}

CR_API cr_status cr_cloud_poll_uploads(cr_cloud *c, int commit, uint32_t *landed_batches,
                                       uint32_t *in_flight_batches) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    uint32_t landed = 0;
    DeviceGuard g(c->ctx->device);
    cr_status st = land(c, false, &landed);
    if (st) return st;
    if (landed_batches) *landed_batches = landed;
    if (in_flight_batches) *in_flight_batches = c->up ? c->up->in_flight_batches : 0;
    if (commit) return flush_mirror(c);
    return CR_OK;
}

CR_API cr_status cr_cloud_wait_uploads(cr_cloud *c, int commit) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    DeviceGuard g(c->ctx->device);
    cr_status st = land(c, true, nullptr);
    if (st) return st;
    if (commit) return flush_mirror(c);
    return CR_OK;
}

CR_API cr_status cr_cloud_set_upload_staging(cr_cloud *c, uint64_t bytes) {
    if (!c) return fail(CR_ERR_INVALID_ARGUMENT, "cloud is null");
    if (bytes < 4096) return fail(CR_ERR_INVALID_ARGUMENT, "staging must be at least 4096 bytes");
    DeviceGuard g(c->ctx->device);
    UploadState &u = state(c);
    cr_status st = land(c, true, nullptr);
    if (st) return st;
    if (u.h_stage) CR_CUDA(cudaFreeHost(u.h_stage));
    u.h_stage = nullptr;
    u.cap = 0;
    u.want_cap = bytes;
    CR_CUDA(cudaHostAlloc((void **)&u.h_stage, bytes, cudaHostAllocDefault));
    u.cap = bytes;
    return CR_OK;
}

}  // extern "C"
