"""The C ABI library without a GPU: it loads, exports every function that
include/pyfwi_b200.h declares, and validates plans on the host."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pyfwi_b200.h")


@pytest.fixture(scope="module")
def native():
    from pyfwi_b200 import build
    build.build()
    from pyfwi_b200 import _native
    return _native


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(pyfwi_\w+)\s*\(", text, re.M)))


def test_exports_every_declared_symbol(native):
    lib = ctypes.CDLL(native.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n


def test_abi_version(native):
    assert native.lib().pyfwi_abi_version() == native.ABI_VERSION == 8


def _geom(native, nz=20, nx=24, npml=4, ns=2, nr=10, half=2):
    g = native.Geometry()
    g.nz, g.nx, g.npml, g.half_order = nz, nx, npml, half
    g.nt, g.nt_ext, g.dt_scale = 50, 50, 1
    g.dt, g.dh = 0.0004, 2.0
    for q, c in enumerate((1.125, -0.041667, 0.0, 0.0)):
        g.c[q] = c
    g.ns, g.nr, g.n_lines = ns, nr, 1
    g.lines[0] = native.RecLine(6, 5, 0, 1, nr, 0, 0)
    g.mask_row0, g.mask_row1, g.mask_col0, g.mask_col1 = 4, nz - 2, 2, nx - 2
    return g


def _create(native, g, opts, srcx=(6, 10), srcz=(6, 6)):
    L = native.lib()
    sx = np.asarray(srcx, np.int32)
    sz = np.asarray(srcz, np.int32)
    h = ctypes.c_void_p()
    rc = L.pyfwi_plan_create(ctypes.byref(g), sx.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                             sz.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(opts), ctypes.byref(h))
    return rc, h


def test_plan_validation(native):
    L = native.lib()
    rc, h = _create(native, _geom(native), native.Options())
    assert rc == 0
    size = ctypes.c_size_t()
    assert L.pyfwi_workspace_size(h, ctypes.byref(size)) == 0 and size.value > 0
    assert L.pyfwi_plan_destroy(h) == 0
    bad = _geom(native, half=3)
    rc, _ = _create(native, bad, native.Options())
    assert rc == -1 and b"half_order" in L.pyfwi_last_error()
    rc, _ = _create(native, _geom(native), native.Options(), srcx=(6, 400))
    assert rc == -1 and b"outside" in L.pyfwi_last_error()
    g = _geom(native)
    g.lines[0] = native.RecLine(6, 5, 1, 1, 10, 0, 0)
    rc, _ = _create(native, g, native.Options())
    assert rc == -1


def test_workspace_grows_with_segment_and_batch(native):
    L = native.lib()
    sizes = {}
    for seg, batch in ((0, 0), (10, 0), (0, 1)):
        o = native.Options()
        o.segment, o.shot_batch = seg, batch
        rc, h = _create(native, _geom(native), o)
        assert rc == 0
        s = ctypes.c_size_t()
        L.pyfwi_workspace_size(h, ctypes.byref(s))
        sizes[(seg, batch)] = s.value
        L.pyfwi_plan_destroy(h)
    assert sizes[(10, 0)] < sizes[(0, 0)]
    assert sizes[(0, 1)] < sizes[(0, 0)]


def test_reverse_mode_needs_sorted_checkpoints(native):
    L = native.lib()
    o = native.Options()
    o.checkpoint = native.CKPT_REVERSE
    chp = np.array([1, 30, 20, 49], np.int32)
    o.nchp, o.chp = 4, chp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    rc, _ = _create(native, _geom(native), o)
    assert rc == -1
    chp = np.array([1, 20, 30, 49], np.int32)
    o.chp = chp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    rc, h = _create(native, _geom(native), o)
    assert rc == 0
    L.pyfwi_plan_destroy(h)


def test_calls_without_workspace_fail_cleanly(native):
    L = native.lib()
    rc, h = _create(native, _geom(native), native.Options())
    assert rc == 0
    assert L.pyfwi_set_model(h, None, 0, None, None, None, None, None, None) == -1
    z = ctypes.c_void_p(1)
    assert L.pyfwi_set_model(h, None, 0, z, z, z, z, z, None) == -2
    L.pyfwi_plan_destroy(h)


def _struct_fields(name):
    text = open(HEADER).read()
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in filter(None, (d.strip() for d in body.split(";"))):
        declarators = re.match(r"(?:const\s+)?\w+\s*\**\s*(.*)$", decl, re.S).group(1)
        names += [re.sub(r"[\s*]|\[\w+\]", "", d) for d in declarators.split(",")]
    return names


@pytest.mark.parametrize("cname,pyname", [("pyfwi_options", "Options"), ("pyfwi_geometry", "Geometry"),
                                          ("pyfwi_rec_line", "RecLine")])
def test_ctypes_structs_follow_the_header(native, cname, pyname):
    """The ctypes mirrors list the header's fields in the header's order."""
    fields = [f[0] for f in getattr(native, pyname)._fields_]
    assert fields == _struct_fields(cname)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without libpyfwi_b200.so there is no compute path: loading raises."""
    from pyfwi_b200 import _native
    monkeypatch.setattr(_native, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_native, "_lib", None)
    with pytest.raises(ImportError):
        _native.lib()
