"""C-ABI checks that need no GPU: the library builds, loads, exports every
symbol include/cr/cr.h declares, and reports the reference's struct layouts."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", "cr", f)
           for f in sorted(os.listdir(os.path.join(ROOT, "include", "cr"))) if f.endswith(".h")]


def declared_symbols():
    names = []
    for h in HEADERS:
        text = open(h).read()
        names += re.findall(r"CR_API\s+[^;(]*?\b(cr_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.fixture(scope="module")
def native(cr):
    import importlib
    build = importlib.import_module("satin-computerasteriser_b200.build")
    build.build()
    from importlib import import_module
    return import_module("satin-computerasteriser_b200._native")


def test_library_exports_every_declared_symbol(native):
    lib = native.lib()
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert missing == []
    # The Python binding declares a prototype for every exported symbol.
    assert sorted(native.PROTOTYPES) == syms


def test_layout_sizes_match_reference(native):
    sizes = (C.c_uint32 * 5)()
    assert native.lib().cr_layout_sizes(sizes) == 0
    assert list(sizes) == [64, 256, 32, 16, 12]
    assert native.BATCH_DTYPE.itemsize == 64
    assert native.FILE_DTYPE.itemsize == 256
    assert native.PIXEL_DTYPE.itemsize == 32
    assert native.VISIBLE_DTYPE.itemsize == 16
    offs = {n: native.BATCH_DTYPE.fields[n][1] for n in native.BATCH_DTYPE.names}
    assert (offs["state"], offs["minX"], offs["maxZ"], offs["numPoints"], offs["firstPoint"],
            offs["fileIndex"]) == (0, 4, 24, 28, 32, 36)


def test_header_compiles_as_c_and_cpp(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "cr/cr.h"\nint main(void){return (int)sizeof(cr_raster_batch)-64;}\n')
    for comp, ext in (("gcc", "c"), ("g++", "cpp")):
        s = tmp_path / f"t.{ext}"
        s.write_text(src.read_text())
        r = subprocess.run([comp, "-std=c11" if ext == "c" else "-std=c++17", "-Wall", "-Werror",
                            "-I", os.path.join(ROOT, "include"), str(s), "-o",
                            str(tmp_path / f"t_{ext}")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert subprocess.run([str(tmp_path / f"t_{ext}")]).returncode == 0


def test_config_defaults_match_swift_defaults(native, cr):
    c = native.cr_config()
    assert native.lib().cr_config_default(C.byref(c)) == 0
    py = cr.ComputeRasteriserConfiguration().to_c()
    for name, _ in native.cr_config._fields_:
        a, b = getattr(c, name), getattr(py, name)
        if name == "backgroundColor":
            assert list(a) == list(b)
        else:
            assert a == b, name
    assert abs(c.depthTolerance - 0.01) < 1e-9 and c.enableCLOD == 1 and c.maximumPointSize == 1.0


def test_status_strings_and_errors_without_device(native, cr):
    lib = native.lib()
    assert lib.cr_status_string(0) == b"CR_OK"
    assert lib.cr_status_string(4) == b"CR_ERR_UNSUPPORTED"
    # Null-handle calls fail cleanly with a detail string.
    assert lib.cr_cloud_commit(None) == 1
    assert b"null" in lib.cr_last_error_detail()
    assert lib.cr_render(None, None, None, 0, None, None) == 1


def test_capacity_preconditions(cr):
    with pytest.raises(cr.CRError):
        cr.ComputeRasteriserCapacity(0)
    with pytest.raises(cr.CRError):
        cr.ComputeRasteriserCapacity(4, 0)
    assert cr.ComputeRasteriserCapacity(3, 10).maxResidentPoints == 30


def test_matrix_multiply_matches_oracle(cr, orc):
    rng = np.random.default_rng(5)
    for _ in range(20):
        a = rng.normal(size=16).astype(np.float32)
        b = rng.normal(size=16).astype(np.float32)
        assert np.array_equal(cr.matrix_multiply(a, b), orc.mat4_mul(a, b))
