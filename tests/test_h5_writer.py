"""The HDF5 writer of the output files (lib/libns2d_h5.so, include/ns2d_h5.h),
checked on CPU with the strict, independently written reader tests/h5read.py:
groups, attributes, the three element types, B-trees of more than one level,
name order, errors, flush-then-append, and the dataset reader."""
import ctypes as C
import os

import numpy as np
import pytest

import h5read

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "2d-navier-stokes_b200", "lib", "libns2d_h5.so")

F64, I32, C128 = 0, 1, 2


@pytest.fixture(scope="module")
def h5():
    if not os.path.exists(LIB):
        pytest.skip("libns2d_h5.so not built (make -C 2d-navier-stokes_b200)")
    L = C.CDLL(LIB)
    L.ns2d_h5_create.restype = C.c_void_p
    L.ns2d_h5_create.argtypes = [C.c_char_p]
    for name in ("ns2d_h5_group", "ns2d_h5_exists"):
        getattr(L, name).argtypes = [C.c_void_p, C.c_char_p]
        getattr(L, name).restype = C.c_int
    L.ns2d_h5_attr_double.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double]
    L.ns2d_h5_dataset.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.c_void_p]
    L.ns2d_h5_flush.argtypes = [C.c_void_p]
    L.ns2d_h5_close.argtypes = [C.c_void_p]
    L.ns2d_h5_error.argtypes = [C.c_void_p]
    L.ns2d_h5_error.restype = C.c_char_p
    L.ns2d_h5_read_double.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_uint64]
    return L


def _ds(L, f, path, a, typ):
    a = np.ascontiguousarray(a)
    dims = (C.c_uint64 * a.ndim)(*a.shape)
    return L.ns2d_h5_dataset(f, path.encode(), typ, a.ndim, dims, a.ctypes.data_as(C.c_void_p))


def test_output_file_layout_round_trip(h5, tmp_path):
    """A Main_HDF_Data-like file: 300 Iter groups (the root's index needs two
    B-tree levels) with TimeValue/TimeStep and real + complex datasets."""
    rng = np.random.default_rng(1)
    fn = str(tmp_path / "main.h5")
    f = h5.ns2d_h5_create(fn.encode())
    assert f
    want = {}
    for it in range(300):
        g = f"/Iter_{it:05d}"
        assert h5.ns2d_h5_group(f, g.encode()) == 0
        assert h5.ns2d_h5_attr_double(f, g.encode(), b"TimeValue", 0.01 * it) == 0
        assert h5.ns2d_h5_attr_double(f, g.encode(), b"TimeStep", 1e-3) == 0
        if it % 50 == 0:
            w = rng.standard_normal((16, 16))
            wh = rng.standard_normal((16, 9)) + 1j * rng.standard_normal((16, 9))
            assert _ds(h5, f, g + "/w", w, F64) == 0
            assert _ds(h5, f, g + "/w_hat", wh, C128) == 0
            want[g + "/w"] = w
            want[g + "/w_hat"] = wh
    assert h5.ns2d_h5_close(f) == 0
    root = h5read.read(fn)
    assert len(root.children) == 300
    assert list(root.children) == sorted(root.children)
    data, attrs = h5read.flatten(root)
    assert set(data) == set(want)
    for k, v in want.items():
        assert data[k].dtype == v.dtype and np.array_equal(data[k], v)
    assert attrs["/Iter_00123"]["TimeValue"].shape == (1,)
    assert float(attrs["/Iter_00123"]["TimeValue"][0]) == 0.01 * 123
    assert float(attrs["/Iter_00007"]["TimeStep"][0]) == 1e-3


def test_types_nesting_and_order(h5, tmp_path):
    fn = str(tmp_path / "misc.h5")
    f = h5.ns2d_h5_create(fn.encode())
    names = ["b", "B", "a_long_name_that_needs_padding", "Z9", "aa", "a"]
    for n in names:
        assert h5.ns2d_h5_group(f, f"/{n}".encode()) == 0
    assert h5.ns2d_h5_group(f, b"/a/inner") == 0
    assert h5.ns2d_h5_group(f, b"/a/inner/deeper") == 0
    assert h5.ns2d_h5_group(f, b"/empty") == 0
    kx = np.arange(-8, 8, dtype=np.int32)
    x = np.linspace(0, 1, 7)
    z = np.zeros((0,))
    cube = np.arange(2 * 3 * 4, dtype=np.float64).reshape(2, 3, 4)
    assert _ds(h5, f, "kx", kx, I32) == 0
    assert _ds(h5, f, "/a/inner/deeper/x", x, F64) == 0
    assert _ds(h5, f, "/a/cube", cube, F64) == 0
    assert _ds(h5, f, "/zero", z, F64) == 0
    assert h5.ns2d_h5_attr_double(f, b"/a/cube", b"scale", 2.5) == 0
    assert h5.ns2d_h5_exists(f, b"/a/inner") == 1 and h5.ns2d_h5_exists(f, b"/nope") == 0
    assert h5.ns2d_h5_close(f) == 0
    root = h5read.read(fn)
    assert list(root.children) == sorted(names + ["empty", "kx", "zero"])
    assert root.children["empty"].children == {}
    data, attrs = h5read.flatten(root)
    assert np.array_equal(data["/kx"], kx) and data["/kx"].dtype == np.int32
    assert np.array_equal(data["/a/inner/deeper/x"], x)
    assert np.array_equal(data["/a/cube"], cube)
    assert data["/zero"].shape == (0,)
    assert float(attrs["/a/cube"]["scale"][0]) == 2.5


def test_errors(h5, tmp_path):
    f = h5.ns2d_h5_create(str(tmp_path / "e.h5").encode())
    one = np.ones(3)
    assert _ds(h5, f, "/missing/x", one, F64) == -1
    assert b"parent" in h5.ns2d_h5_error(f)
    assert _ds(h5, f, "/x", one, F64) == 0
    assert _ds(h5, f, "/x", one, F64) == -1          # exists
    assert h5.ns2d_h5_group(f, b"/x") == -1          # a dataset is there
    assert h5.ns2d_h5_group(f, b"/g") == 0
    assert h5.ns2d_h5_group(f, b"/g") == 0           # existing group: opened
    assert h5.ns2d_h5_attr_double(f, b"/nope", b"a", 1.0) == -1
    assert h5.ns2d_h5_attr_double(f, b"/g", b"a", 1.0) == 0
    assert h5.ns2d_h5_attr_double(f, b"/g", b"a", 2.0) == -1
    assert _ds(h5, f, "/bad", one, 7) == -1
    assert h5.ns2d_h5_close(f) == 0
    assert not h5.ns2d_h5_create(str(tmp_path / "no" / "dir.h5").encode())


def test_flush_then_append(h5, tmp_path):
    """A flushed file is complete; later writes and a second flush supersede it."""
    fn = str(tmp_path / "f.h5")
    f = h5.ns2d_h5_create(fn.encode())
    assert _ds(h5, f, "/a", np.arange(4.0), F64) == 0
    assert h5.ns2d_h5_flush(f) == 0
    data, _ = h5read.flatten(h5read.read(fn))
    assert set(data) == {"/a"}
    assert _ds(h5, f, "/b", np.arange(5.0), F64) == 0
    assert h5.ns2d_h5_close(f) == 0
    data, _ = h5read.flatten(h5read.read(fn))
    assert set(data) == {"/a", "/b"} and np.array_equal(data["/b"], np.arange(5.0))


def test_reader_for_input_files(h5, tmp_path):
    """ns2d_h5_read_double (initial conditions read from file) reads what the
    writer wrote, down nested groups and past a multi-level root index."""
    fn = str(tmp_path / "psi.h5")
    f = h5.ns2d_h5_create(fn.encode())
    for it in range(270):
        assert h5.ns2d_h5_group(f, f"/g{it:04d}".encode()) == 0
    psi = np.random.default_rng(3).standard_normal((32, 32))
    assert _ds(h5, f, "/psi", psi, F64) == 0
    assert _ds(h5, f, "/g0269/psi2", 2 * psi, F64) == 0
    assert _ds(h5, f, "/ints", np.arange(4, dtype=np.int32), I32) == 0
    assert h5.ns2d_h5_close(f) == 0
    out = np.zeros_like(psi)
    assert h5.ns2d_h5_read_double(fn.encode(), b"/psi", out.ctypes.data, out.size) == 0
    assert np.array_equal(out, psi)
    assert h5.ns2d_h5_read_double(fn.encode(), b"/g0269/psi2", out.ctypes.data, out.size) == 0
    assert np.array_equal(out, 2 * psi)
    assert h5.ns2d_h5_read_double(fn.encode(), b"/psi", out.ctypes.data, 10) == -1      # size mismatch
    assert h5.ns2d_h5_read_double(fn.encode(), b"/nothing", out.ctypes.data, out.size) == -1
    assert h5.ns2d_h5_read_double(fn.encode(), b"/ints", out.ctypes.data, 4) == -1      # not doubles
    assert h5.ns2d_h5_read_double(str(tmp_path / "none.h5").encode(), b"/psi", out.ctypes.data, 1) == -1


def test_reader_rejects_corruption(h5, tmp_path):
    """The strict reader notices a damaged file (so the round trips above
    would notice a writer that breaks the format)."""
    fn = str(tmp_path / "c.h5")
    f = h5.ns2d_h5_create(fn.encode())
    for it in range(20):
        h5.ns2d_h5_group(f, f"/Iter_{it:05d}".encode())
    assert h5.ns2d_h5_close(f) == 0
    raw = bytearray(open(fn, "rb").read())
    h5read.read(fn)
    i = raw.find(b"SNOD")
    raw[i + 6] = 9  # claim 9 entries in a node with room for 8
    open(fn, "wb").write(bytes(raw))
    with pytest.raises(h5read.H5FormatError):
        h5read.read(fn)


def test_reader_types_attributes_and_listing(h5, tmp_path):
    """The reading side a post-processor needs: dataset shapes and types,
    complex and int datasets, group attributes, and a group's link names
    (past a multi-level index)."""
    L = h5
    L.ns2d_h5_dataset_info.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_uint64)]
    L.ns2d_h5_read.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_void_p, C.c_uint64]
    L.ns2d_h5_read_attr_double.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_double)]
    L.ns2d_h5_list.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]
    fn = str(tmp_path / "run.h5")
    f = L.ns2d_h5_create(fn.encode())
    rng = np.random.default_rng(9)
    wh = rng.standard_normal((8, 5)) + 1j * rng.standard_normal((8, 5))
    for it in range(300):
        g = f"/Iter_{it:05d}".encode()
        assert L.ns2d_h5_group(f, g) == 0
        assert L.ns2d_h5_attr_double(f, g, b"TimeValue", 0.5 * it) == 0
    assert _ds(L, f, "/Iter_00299/w_hat", wh, C128) == 0
    assert _ds(L, f, "/kx", np.arange(-3, 5, dtype=np.int32), I32) == 0
    assert L.ns2d_h5_close(f) == 0
    t, r, dims = C.c_int(), C.c_int(), (C.c_uint64 * 8)()
    assert L.ns2d_h5_dataset_info(fn.encode(), b"/Iter_00299/w_hat", C.byref(t), C.byref(r), dims) == 0
    assert (t.value, r.value, dims[0], dims[1]) == (C128, 2, 8, 5)
    out = np.zeros((8, 5), dtype=np.complex128)
    assert L.ns2d_h5_read(fn.encode(), b"/Iter_00299/w_hat", C128, out.ctypes.data, out.size) == 0
    assert np.array_equal(out, wh)
    assert L.ns2d_h5_read(fn.encode(), b"/Iter_00299/w_hat", F64, out.ctypes.data, out.size) == -1
    ints = np.zeros(8, dtype=np.int32)
    assert L.ns2d_h5_read(fn.encode(), b"/kx", I32, ints.ctypes.data, 8) == 0
    assert np.array_equal(ints, np.arange(-3, 5))
    v = C.c_double()
    assert L.ns2d_h5_read_attr_double(fn.encode(), b"/Iter_00123", b"TimeValue", C.byref(v)) == 0
    assert v.value == 61.5
    assert L.ns2d_h5_read_attr_double(fn.encode(), b"/Iter_00123", b"Nope", C.byref(v)) == -1
    buf = C.create_string_buffer(1 << 16)
    assert L.ns2d_h5_list(fn.encode(), b"/", buf, len(buf)) == 301
    names = buf.value.decode().split("\n")[:-1]
    assert names == sorted([f"Iter_{i:05d}" for i in range(300)] + ["kx"])
    assert L.ns2d_h5_list(fn.encode(), b"/", buf, 16) == -1  # too small
    assert L.ns2d_h5_list(fn.encode(), b"/kx", buf, len(buf)) == -1  # not a group
