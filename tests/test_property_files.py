"""Property files (INC and GSLIB) against the reference library itself.

The reference's own reader and writers (oracle/_ref/libhpgl.so, built from its
sources) and this library's multi-threaded ones are run on the same arrays and
files: written files must be byte-identical, read values bit-identical with
identical masks, and the same inputs must fail in both.
"""
import ctypes as C
import os

import numpy as np
import pytest

import geo_bsd
import oracle as O
from geo_bsd import hpgl_wrap as W

F32F = np.ctypeslib.ndpointer(dtype="float32", flags=("F", "W", "A"))
U8F = np.ctypeslib.ndpointer(dtype="uint8", flags=("F", "W", "A"))
U8 = np.ctypeslib.ndpointer(dtype="uint8", flags="C")


def _ref():
    if not O.available("ref"):
        pytest.skip("the reference library is not built")
    lib = O.ref_api()
    lib.hpgl_read_inc_file_float.restype = C.c_int
    lib.hpgl_read_inc_file_float.argtypes = [C.c_char_p, C.c_float, C.c_int, F32F, U8F]
    lib.hpgl_read_inc_file_byte.restype = C.c_int
    lib.hpgl_read_inc_file_byte.argtypes = [C.c_char_p, C.c_int, C.c_int, U8F, U8F, U8, C.c_int]
    lib.hpgl_write_inc_file_float.restype = C.c_int
    lib.hpgl_write_inc_file_float.argtypes = [C.c_char_p, C.POINTER(W._HPGL_CONT_MASKED_ARRAY), C.c_float, C.c_char_p]
    lib.hpgl_write_inc_file_byte.restype = C.c_int
    lib.hpgl_write_inc_file_byte.argtypes = [C.c_char_p, C.POINTER(W._HPGL_IND_MASKED_ARRAY), C.c_int, C.c_char_p,
                                             C.POINTER(C.c_ubyte), C.c_int]
    lib.hpgl_write_gslib_cont_property.restype = C.c_int
    lib.hpgl_write_gslib_cont_property.argtypes = [C.POINTER(W._HPGL_CONT_MASKED_ARRAY), C.c_char_p, C.c_char_p,
                                                   C.c_double]
    lib.hpgl_write_gslib_byte_property.restype = C.c_int
    lib.hpgl_write_gslib_byte_property.argtypes = [C.POINTER(W._HPGL_IND_MASKED_ARRAY), C.c_char_p, C.c_char_p,
                                                   C.c_double, C.POINTER(C.c_ubyte), C.c_int]
    return lib


def _cont(data, mask):
    sh = W._HPGL_SHAPE(data=(data.size, 1, 1), strides=(1, data.size, data.size))
    return W._HPGL_CONT_MASKED_ARRAY(data.ctypes.data_as(C.POINTER(C.c_float)), mask.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                     sh)


def _ind(data, mask, count):
    sh = W._HPGL_SHAPE(data=(data.size, 1, 1), strides=(1, data.size, data.size))
    return W._HPGL_IND_MASKED_ARRAY(data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                    mask.ctypes.data_as(C.POINTER(C.c_ubyte)), sh, count)


def _floats(n, seed=1):
    rng = np.random.default_rng(seed)
    d = (rng.lognormal(0, 2, n) * rng.choice([-1, 1], n)).astype(np.float32)
    d[::17] = np.float32(1e-30)
    d[::23] = np.float32(3.4e38)
    d[::29] = np.float32(0.1)
    m = (rng.random(n) < 0.8).astype(np.uint8)
    return d, m


@pytest.mark.parametrize("gslib", [False, True])
def test_float_writers_byte_identical(tmp_path, gslib):
    ref = _ref()
    d, m = _floats(50000)
    a, b = str(tmp_path / "ref.inc"), str(tmp_path / "ours.inc")
    if gslib:
        assert ref.hpgl_write_gslib_cont_property(C.byref(_cont(d, m)), a.encode(), b"PORO", -99.0) == 0
        assert W._hpgl_so.hpgl_write_gslib_cont_property(C.byref(_cont(d, m)), b.encode(), b"PORO", -99.0) == 0
    else:
        assert ref.hpgl_write_inc_file_float(a.encode(), C.byref(_cont(d, m)), -99.0, b"PORO") == 0
        assert W._hpgl_so.hpgl_write_inc_file_float(b.encode(), C.byref(_cont(d, m)), -99.0, b"PORO") == 0
    assert open(a, "rb").read() == open(b, "rb").read()


@pytest.mark.parametrize("gslib", [False, True])
@pytest.mark.parametrize("values", [[10, 20, 200], [7, 8, 9, 10], [5], []])
def test_byte_writers_byte_identical(tmp_path, gslib, values):
    ref = _ref()
    rng = np.random.default_rng(3)
    n = 30000
    d = rng.integers(0, 3, n).astype(np.uint8)
    m = (rng.random(n) < 0.7).astype(np.uint8)
    vals = (C.c_ubyte * max(len(values), 1))(*values)
    a, b = str(tmp_path / "ref.inc"), str(tmp_path / "ours.inc")
    if gslib:
        assert ref.hpgl_write_gslib_byte_property(C.byref(_ind(d, m, 3)), a.encode(), b"FACIES", 255.0, vals,
                                                  len(values)) == 0
        assert W._hpgl_so.hpgl_write_gslib_byte_property(C.byref(_ind(d, m, 3)), b.encode(), b"FACIES", 255.0, vals,
                                                         len(values)) == 0
    else:
        assert ref.hpgl_write_inc_file_byte(a.encode(), C.byref(_ind(d, m, 3)), 255, b"FACIES", vals, len(values)) == 0
        assert W._hpgl_so.hpgl_write_inc_file_byte(b.encode(), C.byref(_ind(d, m, 3)), 255, b"FACIES", vals,
                                                   len(values)) == 0
    assert open(a, "rb").read() == open(b, "rb").read()


FILES = {
    "written": None,  # the reference writer's own output
    "comments": "-- a header comment\n\nPORO values\n1.5 2.5 -- trailing comment\n--x\n 3.25\t4e2\n-99 6 7 8 /\n",
    "crlf": "PORO\r\n1.0\r\n2.0 3.0\r\n4.0 5.0 6.0 7.0 8.0\r\n/\r\n",
    "prefixes": "X\n1.5abc +3 -.5 .25e1 1e-40 0x1p3 inf 8\n",
    "leading": "  3 not a name\n\tPORO\n1 2 3 4 5 6 7 8\n",
    "more_values": "PORO\n1 2 3 4 5 6 7 8 9 10 11 / garbage here\n",
}


def _write(tmp_path, name, text):
    p = str(tmp_path / (name + ".inc"))
    with open(p, "w", newline="") as f:
        f.write(text)
    return p


@pytest.mark.parametrize("case", sorted(FILES))
def test_float_reader_matches_reference(tmp_path, case):
    ref = _ref()
    n = 8
    if FILES[case] is None:
        d, m = _floats(120000, seed=5)
        p = str(tmp_path / "w.inc")
        assert ref.hpgl_write_inc_file_float(p.encode(), C.byref(_cont(d, m)), -99.0, b"PORO") == 0
        n = d.size
    else:
        p = _write(tmp_path, case, FILES[case])
    rd, rm = np.zeros(n, np.float32, order="F"), np.zeros(n, np.uint8, order="F")
    od, om = np.zeros(n, np.float32, order="F"), np.zeros(n, np.uint8, order="F")
    assert ref.hpgl_read_inc_file_float(p.encode(), -99.0, n, rd, rm) == 0
    assert W._hpgl_so.hpgl_read_inc_file_float(p.encode(), -99.0, n, od, om) == 0
    np.testing.assert_array_equal(od.view(np.uint32), rd.view(np.uint32))
    np.testing.assert_array_equal(om, rm)


# (no file here starts with an empty line or ends before its values: the
# reference's reader does not return on those)
@pytest.mark.parametrize("text", ["PORO\n1 2 3 / 4 5 6 7 8\n", "PORO\n1 2 abc 4 5 6 7 8\n", "-- only comments\n"])
def test_float_reader_fails_where_the_reference_fails(tmp_path, text):
    ref = _ref()
    p = _write(tmp_path, "bad", text)
    d, m = np.zeros(8, np.float32, order="F"), np.zeros(8, np.uint8, order="F")
    assert ref.hpgl_read_inc_file_float(p.encode(), -99.0, 8, d, m) == -1
    assert W._hpgl_so.hpgl_read_inc_file_float(p.encode(), -99.0, 8, d, m) == -1
    assert W.last_error()


def test_byte_reader_matches_reference(tmp_path):
    ref = _ref()
    text = "FACIES\n-- comment\n10 20 255 200 20 7 10\n20 200 /\n"
    p = _write(tmp_path, "b", text)
    vals = np.array([10, 20, 200], np.uint8)
    out = []
    for lib in (ref, W._hpgl_so):
        d, m = np.zeros(9, np.uint8, order="F"), np.zeros(9, np.uint8, order="F")
        assert lib.hpgl_read_inc_file_byte(p.encode(), 255, 9, d, m, vals, 3) == 0
        out.append((d.copy(), m.copy()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_geo_round_trip(tmp_path):
    d, m = _floats(64 * 32 * 8, seed=9)
    prop = geo_bsd.ContProperty(d.reshape((64, 32, 8), order="F"), m.reshape((64, 32, 8), order="F"))
    p = str(tmp_path / "rt.inc")
    geo_bsd.write_property(prop, p, "PORO", -99.0)
    back = geo_bsd.load_cont_property(p, -99.0, (64, 32, 8))
    want = np.where(m == 1, d, np.float32(-99.0))
    # %E keeps 7 significant digits; masks survive exactly
    np.testing.assert_array_equal(back.mask, (want != np.float32(-99.0)).astype(np.uint8))
    np.testing.assert_allclose(back.data, want, rtol=1e-6)
    slow = geo_bsd.load_cont_property(p, -99.0)
    np.testing.assert_array_equal(slow.mask, back.mask)
    with pytest.raises(geo_bsd.CriticalValidationError):
        geo_bsd.load_cont_property(str(tmp_path / ".." / "x.inc"), -99.0, 10)
