"""Single-threaded restatement of the reference's PLY loader (test
infrastructure: the checker of the product's parallel parser).

Follows Sources/SatinComputeRasteriser/PLYPointCloudLoader.swift line by
line: parseHeader (:171-240), PLYVertexLayout (:140-158), semantic(for:)
(:160-170), parseASCII (:242-278), parseBinaryLittleEndian (:280-305),
assign / normalizedColor (:307-325), readScalar (:327-352).  Text values are
parsed as Swift's Float(String) does: the token as a C string, no leading
whitespace, libc strtof in the C locale, "snan" as a signalling NaN, and no
value on a range error whose result is infinite or zero.

Returns (positions float32[n, 4] with w = 1, colours float32[n, 4] with
alpha = 1), or raises PLYError(case) with the reference's error case text.
"""
from __future__ import annotations

import ctypes as C
import math
import struct

import numpy as np

TYPES = {"char": ("b", 1, 127.0), "int8": ("b", 1, 127.0),
         "uchar": ("B", 1, 255.0), "uint8": ("B", 1, 255.0),
         "short": ("h", 2, 32767.0), "int16": ("h", 2, 32767.0),
         "ushort": ("H", 2, 65535.0), "uint16": ("H", 2, 65535.0),
         "int": ("i", 4, 2147483647.0), "int32": ("i", 4, 2147483647.0),
         "uint": ("I", 4, 4294967295.0), "uint32": ("I", 4, 4294967295.0),
         "float": ("f", 4, 1.0), "float32": ("f", 4, 1.0),
         "double": ("d", 8, 1.0), "float64": ("d", 8, 1.0)}
SEMANTIC = {"x": "x", "y": "y", "z": "z", "red": "r", "r": "r", "diffuse_red": "r",
            "green": "g", "g": "g", "diffuse_green": "g", "blue": "b", "b": "b",
            "diffuse_blue": "b"}
NEWLINES = "\n\x0b\x0c\r\x85\u2028\u2029"

_libc = C.CDLL(None, use_errno=True)
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.POINTER(C.c_char_p)]


class PLYError(Exception):
    def __init__(self, case: str):
        super().__init__(case)
        self.case = case


def f32(x) -> np.float32:
    return np.float32(x)


def swift_float(token: str):
    """Float(String) (Swift standard library), or None."""
    raw = token.encode("utf-8")
    raw = raw.split(b"\x00", 1)[0]  # a C string ends at NUL
    if not raw or raw[0] in (9, 10, 11, 12, 13, 32):
        return None
    body = raw[1:] if raw[:1] in (b"+", b"-") else raw
    if body.lower() == b"snan":  # Float.signalingNaN bits, sign from the token
        bits = 0xFFA00000 if raw[:1] == b"-" else 0x7FA00000
        return np.array([bits], np.uint32).view(np.float32)[0]
    end = C.c_char_p()
    buf = C.create_string_buffer(raw)
    C.set_errno(0)
    v = _libc.strtof(buf, C.byref(end))
    erange = C.get_errno() == 34
    consumed = C.cast(end, C.c_void_p).value - C.cast(buf, C.c_void_p).value
    if erange and (math.isinf(v) or v == 0.0):
        return None
    if consumed != len(raw):
        return None
    return f32(v)


def split_newlines(text: str) -> list[str]:
    out, cur = [], []
    for ch in text:
        if ch in NEWLINES:
            if cur:
                out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    if cur:
        out.append("".join(cur))
    return out


def parse_header(data: bytes):
    if len(data) < 4:
        raise PLYError("invalidHeader")
    i = data.find(b"end_header")
    if i < 0:
        raise PLYError("invalidHeader")
    end = i + len(b"end_header")
    if end < len(data) and data[end] == 13:
        end += 1
    if end < len(data) and data[end] == 10:
        end += 1
    try:
        text = data[:end].decode("utf-8")
    except UnicodeDecodeError:
        raise PLYError("invalidHeader")
    fmt = count = None
    in_vertex = False
    props = []
    for line in split_newlines(text):
        parts = [p for p in line.split(" ") if p]
        if not parts:
            continue
        k = parts[0]
        if k == "ply":
            continue
        if k == "format":
            if len(parts) < 3:
                raise PLYError("invalidHeader")
            if parts[1] == "ascii":
                fmt = 0
            elif parts[1] == "binary_little_endian":
                fmt = 1
            else:
                raise PLYError(f"unsupportedFormat({parts[1]})")
        elif k == "element":
            if len(parts) < 3:
                raise PLYError("invalidHeader")
            in_vertex = parts[1] == "vertex"
            if in_vertex:
                s = parts[2]
                digits = s[1:] if s[:1] in ("+", "-") else s
                if not digits or not all("0" <= c <= "9" for c in digits):
                    raise PLYError("invalidHeader")
                count = int(s)
                if count < 0 or count > 2 ** 63 - 1:
                    raise PLYError("invalidHeader")
        elif k == "property" and in_vertex:
            if len(parts) < 3:
                raise PLYError("invalidHeader")
            if parts[1] == "list":
                raise PLYError("unsupportedProperty(list " + " ".join(parts[2:]) + ")")
            if parts[1] not in TYPES:
                raise PLYError(f"unsupportedProperty({parts[1]})")
            props.append((parts[2], parts[1]))
    if fmt is None:
        raise PLYError("invalidHeader")
    if count is None:
        raise PLYError("missingVertexElement")
    fields, off = [], 0
    for name, t in props:
        fields.append((SEMANTIC.get(name, None), name, t, off))
        off += TYPES[t][1]
    sems = {f[0] for f in fields}
    if not {"x", "y", "z"} <= sems:
        raise PLYError("missingProperty(x, y, z)")
    return fmt, count, fields, off, end


def _assign(v, field, pos, col):
    sem, _, t, _ = field
    if sem in ("x", "y", "z"):
        pos["xyz".index(sem)] = v
    elif sem in ("r", "g", "b"):
        if t in ("float", "float32", "double", "float64"):
            x = f32(v)
        else:
            x = f32(f32(v) / f32(TYPES[t][2]))
        x = x if x == x else f32(0.0)  # clamp: NaN -> 0
        col["rgb".index(sem)] = min(max(x, f32(0.0)), f32(1.0))


def parse(data: bytes):
    fmt, count, fields, stride, body = parse_header(data)
    pos = np.zeros((count, 4), np.float32)
    col = np.ones((count, 4), np.float32)
    pos[:, 3] = 1.0
    if fmt == 0:
        try:
            text = data[body:].decode("utf-8")
        except UnicodeDecodeError:
            raise PLYError("truncatedBody")
        lines = split_newlines(text)
        if len(lines) < count:
            raise PLYError("truncatedBody")
        for i in range(count):
            values = [v for v in lines[i].split(" ") if v]
            if len(values) < len(fields):
                raise PLYError("truncatedBody")
            for k, field in enumerate(fields):
                v = swift_float(values[k])
                if v is None:
                    raise PLYError(f"invalidASCIIValue(line: {i + 1}, property: {field[1]})")
                _assign(v, field, pos[i], col[i])
    else:
        if body + count * stride > len(data):
            raise PLYError("truncatedBody")
        for i in range(count):
            base = body + i * stride
            for field in fields:
                code, size, _ = TYPES[field[2]]
                raw = struct.unpack_from("<" + code, data, base + field[3])[0]
                v = f32(raw)  # round to nearest float (Float(Int32), Float(Double), ...)
                _assign(v, field, pos[i], col[i])
    return pos, col
