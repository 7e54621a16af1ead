"""PLY input (PLYPointCloudLoader.swift:33-369): the library's parallel
parser against the single-threaded restatement in oracle/ply.py, bit for
bit, on seeded files of every property type, both formats, CRLF / blank
lines / repeated spaces / trailing elements, the float-token edge cases,
every error case (same case text, lowest failing line with many threads),
and the reference's own known-answer test (LayoutTests.swift:44-66).
Host code only: no GPU."""
import importlib
import os

import numpy as np
import pytest

import oracle.ply as oply

TYPES = ["char", "uchar", "short", "ushort", "int", "uint", "float", "double",
         "int8", "uint8", "int16", "uint16", "int32", "uint32", "float32", "float64"]
NP = {"char": "<i1", "int8": "<i1", "uchar": "<u1", "uint8": "<u1", "short": "<i2",
      "int16": "<i2", "ushort": "<u2", "uint16": "<u2", "int": "<i4", "int32": "<i4",
      "uint": "<u4", "uint32": "<u4", "float": "<f4", "float32": "<f4", "double": "<f8",
      "float64": "<f8"}


@pytest.fixture(scope="module")
def cr():
    return importlib.import_module("satin-computerasteriser_b200")


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def random_props(rng):
    """x, y, z (float or double), maybe colours of one random type, extras."""
    ptype = ["float", "double", "float32", "int", "short"][rng.integers(5)]
    props = [("x", ptype), ("y", ptype), ("z", ptype)]
    if rng.random() < 0.85:
        ct = TYPES[rng.integers(len(TYPES))]
        names = [("red", "green", "blue"), ("r", "g", "b"),
                 ("diffuse_red", "diffuse_green", "diffuse_blue")][rng.integers(3)]
        props += [(n, ct) for n in names]
    for k in range(rng.integers(0, 3)):
        props.append((["nx", "alpha", "intensity", "scalar_f"][k], TYPES[rng.integers(len(TYPES))]))
    order = rng.permutation(len(props))
    return [props[i] for i in order]


def values_for(rng, t, n):
    info = np.iinfo(NP[t]) if NP[t][1] in "iu" else None
    if info is not None:
        return rng.integers(info.min, int(info.max) + 1, n, dtype=np.int64).astype(NP[t])
    v = rng.normal(0, 100, n)
    small = rng.random(n) < 0.5  # colour-range values, some outside [0, 1]
    v[small] = rng.uniform(-0.5, 1.5, int(small.sum()))
    return v.astype(NP[t])


def make_ply(rng, n, binary, crlf=False, blank_lines=False, spaces=False, trailing=False):
    props = random_props(rng)
    cols = {name: values_for(rng, t, n) for name, t in props}
    nl = "\r\n" if crlf else "\n"
    head = ["ply", "format " + ("binary_little_endian" if binary else "ascii") + " 1.0",
            "comment seeded fixture", f"element vertex {n}"]
    head += [f"property {t} {name}" for name, t in props]
    if trailing:
        head += ["element face 2", "property list uchar int vertex_indices"]
    head += ["end_header"]
    out = (nl.join(head) + nl).encode()
    if binary:
        rec = np.zeros(n, np.dtype([(name, NP[t]) for name, t in props]))
        for name, _ in props:
            rec[name] = cols[name]
        out += rec.tobytes()
        if trailing:
            out += b"\x03\x00\x00\x00\x00\x01\x00\x00\x00\x02\x00\x00\x00" * 2
        return out
    lines = []
    sep = "  " if spaces else " "
    for i in range(n):
        vals = []
        for name, t in props:
            v = cols[name][i]
            vals.append(repr(float(v)) if NP[t][1] == "f" else str(int(v)))
        lines.append(sep.join(vals) + (" " if spaces and i % 3 == 0 else ""))
        if blank_lines and i % 7 == 3:
            lines.append("")
    body = nl.join(lines)
    if trailing:
        body += nl + "3 0 1 2" + nl + "3 2 1 0"
    return out + body.encode()


@pytest.mark.parametrize("seed", range(12))
def test_parser_matches_oracle_bit_for_bit(cr, seed):
    rng = np.random.default_rng(seed)
    binary = seed % 2 == 1
    data = make_ply(rng, int(rng.integers(1, 1500)), binary, crlf=seed % 3 == 0,
                    blank_lines=seed % 4 == 2, spaces=seed % 5 == 1, trailing=seed % 6 == 0)
    want = oply.parse(data)
    for threads in (1, 3, 16):
        got = cr.PLYPointCloudLoader.parse(data, threads=threads)
        assert same(got[0], want[0]) and same(got[1], want[1]), threads


def test_known_answer_from_reference_layout_tests(cr, orc):
    ply = ("ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n"
           "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\n"
           "end_header\n0 0 0 255 0 0\n1 0 0 0 255 0\n0 1 0 0 0 255").encode()
    pos, col = cr.PLYPointCloudLoader.parse(ply)
    packed = orc.pack(pos[:, :3], colors=col, pointsPerBatch=2)
    assert packed.pointCount == 3
    assert packed.batchCount == 2
    assert {int(c) & 0x00FFFFFF for c in packed.colors} == {0x0000FF, 0x00FF00, 0xFF0000}
    assert len(packed.levels) == 3


TOKENS = ["1e39", "-1e39", "1e-50", "1e-40", "nan", "-inf", "Infinity", "0x1p-3", "+.5", "5.",
          "snan", "-SNaN", "1.0f", "--1", "", "0.1", "3.4028235e38", "3.4028236e38",
          "1.17549435e-38", "7e-46", "1e-45", "00012", "1_0", "٣"]


@pytest.mark.parametrize("tok", TOKENS)
def test_float_tokens(cr, tok):
    data = ("ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\n"
            f"property float z\nend_header\n1 {tok} 2\n").encode()
    try:
        want = oply.parse(data)
    except oply.PLYError as e:
        with pytest.raises(cr.PLYPointCloudLoaderError) as g:
            cr.PLYPointCloudLoader.parse(data)
        assert g.value.case == e.case
        return
    got = cr.PLYPointCloudLoader.parse(data)
    assert same(got[0], want[0]), tok


BAD = {
    "no end_header": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\n",
    "tiny": b"ply",
    "big endian": b"ply\nformat binary_big_endian 1.0\nelement vertex 1\nproperty float x\n"
                  b"property float y\nproperty float z\nend_header\n",
    "no format": b"ply\nelement vertex 1\nproperty float x\nproperty float y\n"
                 b"property float z\nend_header\n1 2 3",
    "no vertex": b"ply\nformat ascii 1.0\nelement face 1\nend_header\n",
    "missing z": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\n"
                 b"property float y\nend_header\n1 2",
    "list": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty list uchar int idx\n"
            b"end_header\n",
    "bad type": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty half x\nend_header\n",
    "bad count": b"ply\nformat ascii 1.0\nelement vertex many\nend_header\n",
    "negative count": b"ply\nformat ascii 1.0\nelement vertex -2\nproperty float x\n"
                      b"property float y\nproperty float z\nend_header\n",
    "short format": b"ply\nformat ascii\nend_header\n",
    "few lines": b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\n"
                 b"property float y\nproperty float z\nend_header\n1 2 3\n4 5 6\n",
    "few values": b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\n"
                  b"property float y\nproperty float z\nend_header\n1 2 3\n4 5\n",
    "bad utf8 body": b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\n"
                     b"property float y\nproperty float z\nend_header\n1 2 \xff\n",
    "bad utf8 header": b"ply\n\xc3\x28\nformat ascii 1.0\nend_header\n",
    "short binary": b"ply\nformat binary_little_endian 1.0\nelement vertex 2\n"
                    b"property float x\nproperty float y\nproperty float z\nend_header\n" + b"\0" * 20,
    "bad value": b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\n"
                 b"property float y\nproperty uchar red\nproperty float z\nend_header\n"
                 b"1 2 3 4\n5 6 seven 8\n",
}


@pytest.mark.parametrize("name", list(BAD))
def test_error_cases_match_the_reference(cr, name):
    data = BAD[name]
    with pytest.raises(oply.PLYError) as e:
        oply.parse(data)
    with pytest.raises(cr.PLYPointCloudLoaderError) as g:
        cr.PLYPointCloudLoader.parse(data, threads=4)
    assert g.value.case == e.value.case, name
    assert str(g.value)  # the reference's errorDescription


def test_lowest_failing_line_wins_with_many_threads(cr):
    rng = np.random.default_rng(7)
    head = ("ply\nformat ascii 1.0\nelement vertex 4000\nproperty float x\nproperty float y\n"
            "property float z\nend_header\n")
    lines = [" ".join(f"{v:.6f}" for v in rng.normal(size=3)) for _ in range(4000)]
    lines[3500] = "1 2 oops"
    lines[2100] = "1 bad 3"
    lines[2999] = "1 2"
    data = (head + "\n".join(lines)).encode()
    for threads in (1, 2, 7, 32):
        with pytest.raises(cr.PLYPointCloudLoaderError) as g:
            cr.PLYPointCloudLoader.parse(data, threads=threads)
        assert g.value.case == "invalidASCIIValue(line: 2101, property: y)"


def test_large_binary_and_ascii_independent_of_threads(cr, tmp_path):
    rng = np.random.default_rng(3)
    n = 300000
    rec = np.zeros(n, np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("red", "u1"),
                                ("green", "u1"), ("blue", "u1"), ("alpha", "u1")]))
    for f in ("x", "y", "z"):
        rec[f] = rng.normal(0, 50, n)
    for f in ("red", "green", "blue", "alpha"):
        rec[f] = rng.integers(0, 256, n)
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\nproperty float x\n"
            "property float y\nproperty float z\nproperty uchar red\nproperty uchar green\n"
            "property uchar blue\nproperty uchar alpha\nend_header\n" % n).encode()
    path = os.path.join(tmp_path, "big.ply")
    with open(path, "wb") as f:
        f.write(head + rec.tobytes())
    a = cr.PLYPointCloudLoader.read(path, threads=1)
    b = cr.PLYPointCloudLoader.read(path, threads=12)
    assert same(a[0], b[0]) and same(a[1], b[1])
    assert np.array_equal(a[0][:, 0], rec["x"]) and np.array_equal(a[0][:, 2], rec["z"])
    assert np.array_equal(a[1][:, 1], (rec["green"].astype(np.float32) / np.float32(255)))
    assert (a[1][:, 3] == 1).all()
    m = 60000
    text = head.replace(b"binary_little_endian", b"ascii").replace(b"%d" % n, b"%d" % m)
    body = "\n".join(f"{float(rec['x'][i])!r} {float(rec['y'][i])!r} {float(rec['z'][i])!r} "
                     f"{rec['red'][i]} "
                     f"{rec['green'][i]} {rec['blue'][i]} {rec['alpha'][i]}"
                     for i in range(m)).encode()
    a = cr.PLYPointCloudLoader.parse(text + body, threads=1)
    b = cr.PLYPointCloudLoader.parse(text + body, threads=9)
    assert same(a[0], b[0]) and same(a[1], b[1])
    assert np.array_equal(a[0][:, 1], rec["y"][:m])
    prefix = body[:body.index(b"\n", 200000)]  # the oracle on the first k lines
    k = prefix.count(b"\n") + 1
    want = oply.parse(text.replace(b"vertex %d" % m, b"vertex %d" % k) + prefix)
    assert k > 1000 and same(a[0][:k], want[0]) and same(a[1][:k], want[1])


def test_empty_and_missing_files(cr, tmp_path):
    empty = os.path.join(tmp_path, "empty.ply")
    open(empty, "wb").close()
    with pytest.raises(cr.PLYPointCloudLoaderError) as g:
        cr.PLYPointCloudLoader.read(empty)
    assert g.value.case == "invalidHeader"
    with pytest.raises(cr.CRError):
        cr.PLYPointCloudLoader.read(os.path.join(tmp_path, "nope.ply"))
    zero = b"ply\nformat ascii 1.0\nelement vertex 0\nproperty float x\nproperty float y\n" \
           b"property float z\nend_header\n"
    pos, col = cr.PLYPointCloudLoader.parse(zero)
    assert pos.shape == (0, 4) and col.shape == (0, 4)
