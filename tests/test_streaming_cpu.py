"""StreamingAdapter (StreamingAdapter.swift:17-200) on the host, against a
model of the slot pool whose asynchronous uploads land a few ticks late.

Checks the reference harness's invariants
(StreamingResidencyIntegrationTests.swift:330-380) over a scripted camera
path (far, zoom, orbit, hold) through a deliberately undersized pool:
* pool pressure happens (the source wants more than the pool holds);
* no leak: every chunk the source counts as resident is resident in the
  adapter or still queued, every tick, and the hold phase ends with none;
* residentPoints mirrors the cloud's point count every tick;
* queued chunks drain once evictions free slots, and freed slots are reused;
plus the two drop paths: a chunk wider than the whole pool, and a queued
chunk evicted before its upload.
"""
import importlib

import numpy as np
import pytest

from scenes import blob_cloud


@pytest.fixture(scope="module")
def streaming():
    return importlib.import_module("satin-computerasteriser_b200.streaming")


class PoolModel:
    """The slot pool's bookkeeping with asynchronous uploads: slots taken at
    once, published `lag` polls later, cancelled if removed in flight."""

    def __init__(self, slots: int, lag: int = 2):
        self.batchCount = slots
        self.free = list(range(slots - 1, -1, -1))
        self.resident = {}          # slot -> points
        self.flight = []            # [ticks_left, [(slot, points)]]
        self.cancelled = set()
        self.lag = lag
        self.assigned_history = []
        self.commits = 0

    @property
    def freeSlotCount(self):
        return len(self.free)

    @property
    def pointCount(self):
        return sum(self.resident.values())

    def addBatchesAsync(self, low, med, high, colors, levels, batches, borrow=False):
        assert len(batches) <= len(self.free)
        slots = [self.free.pop() for _ in range(len(batches))]
        self.assigned_history.extend(slots)
        self.flight.append([self.lag, list(zip(slots, batches["numPoints"].tolist()))])
        return slots

    def removeBatches(self, slots, commit=True):
        flying = {s for _, sl in self.flight for s, _ in sl}
        for s in slots:
            if s in flying:
                self.cancelled.add(s)
            elif s in self.resident:
                del self.resident[s]
                self.free.append(s)

    def pollUploads(self, commit=True):
        landed = 0
        for f in self.flight:
            f[0] -= 1
        while self.flight and self.flight[0][0] <= 0:
            _, sl = self.flight.pop(0)
            for s, n in sl:
                landed += 1
                if s in self.cancelled:
                    self.cancelled.discard(s)
                    self.free.append(s)
                else:
                    self.resident[s] = n
        return landed, sum(len(sl) for _, sl in self.flight)

    def commitBatchUpdates(self):
        self.commits += 1


class Cam:
    def __init__(self, pos, target):
        import importlib as il
        cr = il.import_module("satin-computerasteriser_b200")
        self.c = cr.PerspectiveCamera(position=tuple(pos), near=0.01, far=100.0, fov=45.0,
                                      aspect=16 / 9)
        self.c.lookAt(tuple(target))

    @property
    def position(self):
        return self.c.position

    @property
    def viewMatrix(self):
        return self.c.viewMatrix

    @property
    def projectionMatrix(self):
        return self.c.projectionMatrix


def test_adapter_invariants_under_pool_pressure(orc, streaming):
    pos, rgba = blob_cloud(160000, 44)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=512)
    chunks = streaming.chunks_from_packed(packed, 4)
    assert len(chunks) > 60
    src = streaming.InMemoryStreamingSource(chunks, budget_bytes=160 * 512 * 17)
    pool = PoolModel(slots=96, lag=2)
    ad = streaming.StreamingAdapter(src, pool)
    ad.maxChunkUploadsPerTick = 8
    recs = []

    def tick(phase, cam):
        ad.update(cam, (1920, 1080))
        believed = len(src.believed)
        recs.append(dict(phase=phase, believed=believed, resident=ad.residentChunks,
                         pending=ad.pendingUploadCount, full=ad.lastError is not None,
                         pts=ad.residentPoints, cloud_pts=pool.pointCount))

    for i in range(12):
        tick("far", Cam((0, 0, 3.0), (0, 0, 0)))
    for i in range(12):
        tick("zoom", Cam((0.45, 0.45, 0.7), (0.4, 0.4, 0.0)))
    for i in range(18):
        a = 2 * np.pi * i / 18
        tick("orbit", Cam((1.2 * np.cos(a), 0.3, 1.2 * np.sin(a)), (0, 0, 0)))
    hold = len(recs)
    for i in range(12):
        tick("hold", Cam((1.2, 0.3, 0.0), (0, 0, 0)))

    assert max(r["believed"] for r in recs) * 4 > pool.batchCount or any(r["full"] for r in recs)
    assert any(r["full"] for r in recs)
    for r in recs:
        assert r["believed"] - r["resident"] - r["pending"] == 0, r
        assert r["pts"] == r["cloud_pts"], r
    # Over-subscribed: chunks stay queued while the pool is full, and the
    # held camera settles (no churn in the resident set).
    assert any(r["pending"] > 0 for r in recs[:hold])
    assert len({(r["resident"], r["pending"]) for r in recs[hold + 4:]}) == 1
    # Slots were reused after evictions.
    assert len(pool.assigned_history) > len(set(pool.assigned_history))
    # Resident slots hold exactly the resident chunks' batches.
    ad.update(Cam((1.2, 0.3, 0.0), (0, 0, 0)), (1920, 1080))
    for _ in range(4):
        pool.pollUploads()
    want = sum(len(c.batches) for c in chunks if c.id in ad.slotsByChunk)
    assert len(pool.resident) == want


def test_oversize_chunk_is_dropped_and_evicted_queued_chunk_is_not_uploaded(orc, streaming):
    pos, rgba = blob_cloud(40000, 5)
    packed = orc.pack(pos, colors_rgba8=rgba, pointsPerBatch=512)
    big = streaming.chunks_from_packed(packed, 12)[0]
    small = streaming.chunks_from_packed(packed, 2)[:3]
    pool = PoolModel(slots=8, lag=1)

    class Scripted:
        def __init__(self, updates):
            self.updates = list(updates)
            self.believed = set()

        def submit(self, view):
            pass

        def pollLatest(self):
            if not self.updates:
                return None
            u = self.updates.pop(0)
            for cid in u.removed:
                self.believed.discard(cid)
            for c in u.added:
                self.believed.add(c.id)
            return u

        def setBudget(self, n):
            pass

        def close(self):
            pass

    small = [streaming.ResidentChunk(streaming.ChunkID(1, i, 0, 0), c.batches, c.xyzLow,
                                     c.xyzMed, c.xyzHigh, c.colors, c.levels)
             for i, c in enumerate(small)]
    U = streaming.StreamingUpdate
    src = Scripted([U([big] + small, []), U([], [small[2].id])])
    ad = streaming.StreamingAdapter(src, pool)
    ad.maxChunkUploadsPerTick = 2
    cam = Cam((0, 0, 3.0), (0, 0, 0))
    ad.update(cam, (640, 480))
    assert "pool capacity" in ad.lastError  # 12 batches > 8 slots: dropped
    assert big.id not in ad.slotsByChunk
    assert set(ad.slotsByChunk) == {small[0].id, small[1].id}
    assert ad.pendingUploadCount == 1  # small[2] queued by the per-tick cap
    ad.update(cam, (640, 480))          # small[2] evicted while queued
    assert ad.pendingUploadCount == 0
    assert small[2].id not in ad.slotsByChunk
    for _ in range(3):
        ad.update(cam, (640, 480))
    assert ad.residentPoints == sum(c.totalPointCount for c in small[:2])


def test_pixel_scale_matches_reference_formula(streaming):
    p = np.zeros(16, np.float32)
    p[5] = 1.0 / np.tan(np.radians(30.0))
    assert streaming.screen_space_pixel_scale(1080.0, p) == pytest.approx(540.0 * p[5])
