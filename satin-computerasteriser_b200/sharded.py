"""One frame whose points are split over the ranks of a process group.

Each rank (one process per GPU) holds a part of the cloud's batches — a
contiguous range of the packed batch list (``shard_range``) — and renders the
same camera into a frame of the same size.  The HQS passes then compose
across ranks through two integer reductions:

1. every rank runs the depth stage (clear, cull, depth pass) over its batches;
2. the depth planes are combined by an element-wise maximum (all-reduce):
   the reverse-Z depth of the nearest point of ANY rank, which is the depth
   plane of the whole cloud, because max is associative and commutative;
3. every rank runs the colour stage over its batches against that depth;
4. the R, G, B, count planes are summed (all-reduce);
5. every rank resolves (and hole-fills) the summed planes.

Integer max and sum do not depend on the order, so every rank's image is
bit-identical to one ``encode()`` of the whole cloud on one GPU.  There is
no counterpart in the reference (Metal, one GPU).

The collectives are torch.distributed all-reduces: NCCL over NVLink for
device planes, or gloo for host planes (the CPU tests run the same flow on
planes that the oracle produces).  NCCL's signed 32-bit max would misorder
depths of 2^31 and above, so the depth plane is flipped into signed order
(top bit XORed, ``cr_frame_flip_depth_order``) around the maximum.  The sum
of 32-bit fields is the same bits as signed or unsigned.
"""
from __future__ import annotations

STAGE_DEPTH, STAGE_COLOR, STAGE_RESOLVE = 1, 2, 4


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """The contiguous part [lo, hi) of n items that rank `rank` of `world` holds
    (sizes differ by at most one; every item in exactly one part)."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("need 0 <= rank < world and n >= 0")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def render_point_sharded(run_stage, depth_i32, accum_i32, flip_depth, group=None):
    """The stage / collective sequence of one frame split by points.

    run_stage(stages)  runs stages of this rank's part (cr_render_stages)
    depth_i32          the frame's depth plane viewed as int32 (a tensor)
    accum_i32          the frame's R, G, B, count planes viewed as int32
    flip_depth()       XORs the top bit of every depth word in place
    Every rank calls this with the same frame size and camera, in the same
    order with respect to its other collectives."""
    import torch.distributed as dist

    run_stage(STAGE_DEPTH)
    flip_depth()
    dist.all_reduce(depth_i32, op=dist.ReduceOp.MAX, group=group)
    flip_depth()
    run_stage(STAGE_COLOR)
    dist.all_reduce(accum_i32, op=dist.ReduceOp.SUM, group=group)
    run_stage(STAGE_RESOLVE)


class _DevicePlane:
    """A device allocation described with the CUDA array interface (v3) for
    torch.as_tensor; the frame owns the memory."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


class PointShardedRasteriser:
    """encode() of a ComputeRasteriser whose clouds hold this rank's part of the
    batches, composed with the other ranks' parts over a NCCL process group.

    All ranks call encode() for every frame with the same camera and viewport
    (update / resize as usual on the wrapped rasteriser).  After encode() the
    wrapped rasteriser's outputs (outputRGBA8, depthTexture, pixels) hold the
    whole cloud's image on every rank.  HQS only."""

    def __init__(self, rasteriser, group=None):
        self.rasteriser = rasteriser
        self.group = group

    def encode(self):
        import torch

        r = self.rasteriser
        pl = r.devicePlanes()
        dev = torch.device("cuda", pl["device"])
        depth = torch.as_tensor(_DevicePlane(pl["depth"], pl["pixels"]), device=dev)
        accum = torch.as_tensor(_DevicePlane(pl["accum"], 4 * pl["pixels"]), device=dev)
        # The collectives are ordered with the library's stream: NCCL waits
        # for the depth / colour stages enqueued before it, and the next
        # stage waits for the all-reduce.
        stream = torch.cuda.ExternalStream(pl["stream"], device=dev)
        with torch.cuda.stream(stream):
            render_point_sharded(r.encodeStages, depth, accum, r.flipDepthOrder, self.group)
