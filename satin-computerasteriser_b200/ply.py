"""PLY input: PLYPointCloudLoader (PLYPointCloudLoader.swift:33-369).

The parser is the library's (``cr_ply_parse``, C++ on every host core); it
yields the float4 positions and colours that the reference hands to its CPU
packer, and ``load`` packs them on the GPU (``GPUPacker.pack``) into a slot
pool.  Errors raise PLYPointCloudLoaderError with the reference's case
(``.case``) and message (errorDescription, :13-30).
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

from . import _native as N

ASCII, BINARY_LITTLE_ENDIAN = 0, 1

_MESSAGES = [
    (r"invalidHeader", lambda m: "The file is not a valid PLY file."),
    (r"unsupportedFormat\((.*)\)", lambda m: f"Unsupported PLY format: {m.group(1)}."),
    (r"missingVertexElement", lambda m: "The PLY file does not contain a vertex element."),
    (r"missingProperty\((.*)\)",
     lambda m: f"The PLY file is missing required property '{m.group(1)}'."),
    (r"unsupportedProperty\((.*)\)",
     lambda m: f"Unsupported PLY vertex property '{m.group(1)}'."),
    (r"truncatedBody", lambda m: "The PLY file ended before all vertex data could be read."),
    (r"invalidASCIIValue\(line: (\d+), property: (.*)\)",
     lambda m: f"Could not parse property '{m.group(2)}' on vertex line {m.group(1)}."),
]


class PLYPointCloudLoaderError(Exception):
    """PLYPointCloudLoaderError (PLYPointCloudLoader.swift:4-30): `case` is the
    enum case as text, e.g. "invalidASCIIValue(line: 3, property: y)"."""

    def __init__(self, case: str):
        self.case = case
        msg = case
        for pat, fn in _MESSAGES:
            m = re.fullmatch(pat, case)
            if m:
                msg = fn(m)
                break
        super().__init__(msg)


def _check(st: int):
    if st == 9:  # CR_ERR_FORMAT
        raise PLYPointCloudLoaderError(N.last_error_detail())
    N.check(st)


class PLYPointCloudLoader:
    """PLYPointCloudLoader: parse(data) / read(path) give the vertices as
    (positions float32[n, 4], colours float32[n, 4]); load(context, path)
    packs them on the GPU into a ComputeRasteriserPointCloud."""

    @staticmethod
    def header(data) -> dict:
        buf = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
        h = N.cr_ply_header()
        _check(N.lib().cr_ply_read_header(N.ptr(buf), buf.size, C.byref(h)))
        return {"vertexCount": h.vertexCount, "bodyOffset": h.bodyOffset,
                "format": h.format, "propertyCount": h.propertyCount, "stride": h.stride,
                "colorProperties": h.colorProperties}

    @staticmethod
    def _parse_ptr(ptr, size: int, threads: int):
        h = N.cr_ply_header()
        _check(N.lib().cr_ply_read_header(ptr, size, C.byref(h)))
        n = int(h.vertexCount)
        pos = np.empty((n, 4), np.float32)
        col = np.empty((n, 4), np.float32)
        _check(N.lib().cr_ply_parse(ptr, size, int(threads), N.ptr(pos), N.ptr(col)))
        return pos, col

    @staticmethod
    def parse(data, threads: int = 0):
        """parse(_:pointsPerBatch:)'s vertex step on bytes in memory."""
        buf = np.frombuffer(data, np.uint8) if not isinstance(data, np.ndarray) else data
        buf = np.ascontiguousarray(buf)
        return PLYPointCloudLoader._parse_ptr(N.ptr(buf), buf.size, threads)

    @staticmethod
    def read(path: str | os.PathLike, threads: int = 0):
        """load(url:)'s vertex step: the file is mapped, not read into memory."""
        data, size = C.c_void_p(), C.c_uint64()
        _check(N.lib().cr_file_map(os.fsencode(path), C.byref(data), C.byref(size)))
        try:
            return PLYPointCloudLoader._parse_ptr(data, size.value, threads)
        finally:
            N.lib().cr_file_unmap(data, size)

    @staticmethod
    def load(context, path: str | os.PathLike, pointsPerBatch: int = 128 * 80, into=None,
             packer=None, threads: int = 0):
        """load(url:pointsPerBatch:) with the GPU packer: the file's points packed
        (Morton order, LOD levels, split-precision words, float colours
        truncated to 8 bits as the reference's pack) into `into` or a new
        cloud of ceil(n / pointsPerBatch) slots."""
        from . import ComputeRasteriserCapacity, ComputeRasteriserPointCloud, GPUPacker
        pos, col = PLYPointCloudLoader.read(path, threads)
        n = len(pos)
        if into is None:
            nb = max(1, (n + pointsPerBatch - 1) // pointsPerBatch)
            into = ComputeRasteriserPointCloud(context,
                                               ComputeRasteriserCapacity(nb, pointsPerBatch))
        (packer or GPUPacker(context)).pack(positions=pos, colors=col, count=n, into=into)
        return into
