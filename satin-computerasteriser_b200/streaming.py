"""Streaming residency: a slot pool fed chunk by chunk as the camera moves.

Mirrors the reference's streaming layer
(Sources/SatinComputeRasteriserStreaming/StreamingAdapter.swift:17-200):

  StreamingPointCloudSource   the source protocol the adapter drives
                              (SwiftPDAL's StreamingPointCloudSource: submit a
                              camera view, poll the latest residency delta)
  StreamingAdapter            per frame: submit the view, drain the delta,
                              free evicted slots, upload up to
                              maxChunkUploadsPerTick queued chunks, commit once
  InMemoryStreamingSource     a source over chunks held in host memory, with
                              the distance-only residency policy (nearest
                              chunks first, up to a byte budget)

The reference's source reads COPC files through PDAL / lazperf, which are
not part of this build; any object with the protocol's methods plugs in.

Difference from the reference: uploads are asynchronous
(``addBatchesAsync``).  A chunk's slots are taken when it is uploaded, and it
counts as resident from then on (``residentChunks``), but its points are
drawn only after the copy has landed and a later ``update`` published it
(``ComputeRasteriserPointCloud.pollUploads``).  So the copy never stalls the
frame that enqueued it.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import NamedTuple, Protocol

import numpy as np

from ._native import BATCH_DTYPE

BYTES_PER_POINT = 17  # xyzLow + xyzMed + xyzHigh + colors (4 B each) + level (1 B)


class ChunkID(NamedTuple):
    """A chunk's key (COPC octree node: depth and cell; any hashable works)."""
    depth: int
    x: int
    y: int
    z: int


@dataclass
class ResidentChunk:
    """One chunk's packed points: batches (BATCH_DTYPE, firstPoint into these
    arrays, level-ascending with cumulative LOD counts) and the split-
    precision words, colours and levels."""
    id: ChunkID
    batches: np.ndarray
    xyzLow: np.ndarray
    xyzMed: np.ndarray
    xyzHigh: np.ndarray
    colors: np.ndarray
    levels: np.ndarray
    pinned: bool = False  # arrays in page-locked memory (pin_chunks): uploads borrow them

    @property
    def totalPointCount(self) -> int:
        return len(self.levels)

    @property
    def bounds(self) -> tuple[np.ndarray, np.ndarray]:
        b = self.batches
        lo = np.array([b["minX"].min(), b["minY"].min(), b["minZ"].min()], np.float64)
        hi = np.array([b["maxX"].max(), b["maxY"].max(), b["maxZ"].max()], np.float64)
        return lo, hi


@dataclass
class StreamingUpdate:
    added: list = field(default_factory=list)    # ResidentChunk
    removed: list = field(default_factory=list)  # ChunkID


@dataclass
class StreamingCameraView:
    position: np.ndarray
    viewProjection: np.ndarray  # column-major float32[16]
    pixelScale: float


class StreamingPointCloudSource(Protocol):
    def submit(self, view: StreamingCameraView) -> None: ...
    def pollLatest(self) -> StreamingUpdate | None: ...
    def setBudget(self, nbytes: int) -> None: ...
    def close(self) -> None: ...


def screen_space_pixel_scale(viewport_height: float, projection) -> float:
    """ComputeRasteriserProjection.screenSpacePixelScale (ProjectionHelpers.swift:36-42):
    viewportHeight * 0.5 * projectionMatrix[1][1] (column-major element 5)."""
    p = np.asarray(projection, np.float32).reshape(-1)
    return float(np.float32(viewport_height) * np.float32(0.5) * p[5])


def chunks_from_packed(packed, batches_per_chunk: int) -> list[ResidentChunk]:
    """Consecutive runs of a packed cloud's batches (Morton order, so each run
    is a compact region) as chunks with their own arrays."""
    out = []
    nb = len(packed.batches)
    for k, b0 in enumerate(range(0, nb, batches_per_chunk)):
        bs = np.array(packed.batches[b0:b0 + batches_per_chunk], dtype=BATCH_DTYPE)
        p0 = int(bs["firstPoint"][0])
        p1 = int(bs["firstPoint"][-1]) + int(bs["numPoints"][-1])
        bs["firstPoint"] -= p0
        out.append(ResidentChunk(ChunkID(0, k, 0, 0), bs,
                                 np.array(packed.xyzLow[p0:p1]), np.array(packed.xyzMed[p0:p1]),
                                 np.array(packed.xyzHigh[p0:p1]), np.array(packed.colors[p0:p1]),
                                 np.array(packed.levels[p0:p1])))
    return out


def pin_chunks(chunks: list[ResidentChunk]):
    """Moves the chunks' arrays into one page-locked host arena (HostBuffer) so
    that uploads read them directly (addBatchesAsync(borrow=True), no staging
    copy).  Returns the arena, which must outlive every upload from it."""
    from . import HostBuffer

    def a16(x):
        return (x + 15) & ~15
    total = sum(4 * a16(4 * c.totalPointCount) + a16(c.totalPointCount) for c in chunks)
    arena = HostBuffer((max(total, 16),), np.uint8)
    buf, off = arena.array, 0
    for c in chunks:
        n = c.totalPointCount
        for name in ("xyzLow", "xyzMed", "xyzHigh", "colors"):
            view = buf[off:off + 4 * n].view(np.uint32)
            view[:] = getattr(c, name)
            setattr(c, name, view)
            off += a16(4 * n)
        lv = buf[off:off + n]
        lv[:] = c.levels
        c.levels = lv
        off += a16(n)
        c.pinned = True
    return arena


class InMemoryStreamingSource:
    """A streaming source over chunks in host memory.

    Residency policy (distance only): on each submitted view the chunks are
    ranked by the distance from the camera to their bounding-box centre, and
    the nearest ones are wanted while their points fit the byte budget
    (BYTES_PER_POINT per point).  pollLatest returns what entered and left the
    wanted set since the last poll, and then counts the added chunks as
    resident on the GPU (the model the adapter must keep up with)."""

    def __init__(self, chunks: list[ResidentChunk], budget_bytes: int, pin: bool = False):
        # pin: chunks in one page-locked arena, uploaded without a staging copy
        # (the source must then outlive the uploads from it).
        self._arena = pin_chunks(chunks) if pin else None
        self.chunks = {c.id: c for c in chunks}
        self._ids = list(self.chunks)
        self._centres = np.array([0.5 * (c.bounds[0] + c.bounds[1]) for c in chunks],
                                 np.float64).reshape(-1, 3)
        self._cost = np.array([c.totalPointCount * BYTES_PER_POINT for c in chunks], np.int64)
        self.budget = int(budget_bytes)
        self.believed: set = set()
        self._wanted: list = []
        self.closed = False

    def setBudget(self, nbytes: int):
        self.budget = int(nbytes)

    def submit(self, view: StreamingCameraView):
        pos = np.asarray(view.position, np.float64)
        d = np.linalg.norm(self._centres - pos, axis=1)
        order = np.argsort(d, kind="stable")  # ties: chunk order
        fits = np.cumsum(self._cost[order]) <= self.budget
        n = len(order) if fits.all() else int(np.argmin(fits))  # nearest prefix in budget
        self._wanted = [self._ids[i] for i in order[:n]]

    def pollLatest(self) -> StreamingUpdate | None:
        if self.closed:
            return None
        want = set(self._wanted)
        removed = [i for i in sorted(self.believed) if i not in want]
        added = [self.chunks[i] for i in self._wanted if i not in self.believed]
        if not removed and not added:
            return None
        self.believed = want
        return StreamingUpdate(added, removed)

    def close(self):
        self.closed = True


class StreamingAdapter:
    """Bridges a streaming source to a ComputeRasteriserPointCloud slot pool
    (StreamingAdapter.swift:17-200).

    Per ``update(camera, viewport)``: publish the uploads that have landed,
    submit the camera view, drain the source's delta, free evicted chunks'
    slots (dropping queued chunks evicted before their upload), upload up to
    ``maxChunkUploadsPerTick`` queued chunks, and commit the batch table once.
    A chunk that does not fit the free slots stays queued (back-pressure) and
    ``lastError`` says so; a chunk wider than the whole pool is dropped.
    Invariant: every chunk the source counts as resident is either resident
    here (slots assigned) or queued (``pendingUploadCount``)."""

    def __init__(self, source, cloud):
        self.source = source
        self.cloud = cloud
        self.slotsByChunk: dict = {}
        self.pendingAdds: list = []
        self.pendingCursor = 0
        self.residentChunks = 0
        self.residentPoints = 0
        self.lastError: str | None = None
        self.maxChunkUploadsPerTick = 4

    @property
    def pendingUploadCount(self) -> int:
        return len(self.pendingAdds) - self.pendingCursor

    def setBudget(self, nbytes: int):
        self.source.setBudget(nbytes)

    def update(self, camera, viewport):
        """One tick (StreamingAdapter.swift:71-177)."""
        landed, _ = self.cloud.pollUploads(commit=False)
        dirty = landed > 0
        vp = np.asarray(viewport, np.float32).reshape(-1)
        proj = np.asarray(camera.projectionMatrix, np.float32).reshape(-1)
        view = np.asarray(camera.viewMatrix, np.float32).reshape(-1)
        from . import matrix_multiply
        self.source.submit(StreamingCameraView(
            position=np.asarray(camera.position, np.float64),
            viewProjection=matrix_multiply(proj, view),
            pixelScale=screen_space_pixel_scale(float(vp[-1]), proj)))
        delta = self.source.pollLatest()
        if delta is None and self.pendingCursor >= len(self.pendingAdds):
            if dirty:
                self.cloud.commitBatchUpdates()
            self._refresh()
            return
        if delta is not None:
            slots_to_free = []
            for cid in delta.removed:
                slots = self.slotsByChunk.pop(cid, None)
                if slots is not None:
                    slots_to_free.extend(slots)
            if delta.removed:
                # Queued chunks evicted before their upload are dropped.
                if self.pendingCursor > 0:
                    del self.pendingAdds[:self.pendingCursor]
                    self.pendingCursor = 0
                gone = set(delta.removed)
                self.pendingAdds = [c for c in self.pendingAdds if c.id not in gone]
            if slots_to_free:
                self.cloud.removeBatches(slots_to_free, commit=False)
                dirty = True
            self.pendingAdds.extend(delta.added)
        uploaded = 0
        while uploaded < self.maxChunkUploadsPerTick and self.pendingCursor < len(self.pendingAdds):
            chunk = self.pendingAdds[self.pendingCursor]
            need = len(chunk.batches)
            if self.cloud.freeSlotCount < need:
                if need > self.cloud.batchCount:
                    self.lastError = (f"chunk needs {need} slots but pool capacity is "
                                      f"{self.cloud.batchCount}; raise maxResidentBatches")
                    self.pendingCursor += 1
                    continue
                # Pool full for now: keep the chunk at the cursor for a later
                # tick (an eviction frees slots) and stop draining this tick.
                self.lastError = (f"slot pool full (capacity {self.cloud.batchCount}); raise "
                                  "budget or maxResidentBatches")
                break
            self.pendingCursor += 1
            slots = self.cloud.addBatchesAsync(chunk.xyzLow, chunk.xyzMed, chunk.xyzHigh,
                                               chunk.colors, chunk.levels, chunk.batches,
                                               borrow=chunk.pinned)
            self.slotsByChunk[chunk.id] = slots
            dirty = True
            uploaded += 1
        if self.pendingCursor == len(self.pendingAdds):
            self.pendingAdds.clear()
            self.pendingCursor = 0
        elif self.pendingCursor > 64 and self.pendingCursor * 2 > len(self.pendingAdds):
            del self.pendingAdds[:self.pendingCursor]
            self.pendingCursor = 0
        if dirty:
            self.cloud.commitBatchUpdates()
        self._refresh()

    def _refresh(self):
        self.residentChunks = len(self.slotsByChunk)
        self.residentPoints = self.cloud.pointCount

    def close(self):
        self.pendingAdds.clear()
        self.pendingCursor = 0
        self.source.close()
