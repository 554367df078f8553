"""The serial package's data-array file format (lsm_data_arrays.c:363-435):
three native ints (ghost-box dims) then the values, x fastest; gzip/bzip2
compression by name."""
import os

import numpy as np
import pytest
import torch

from pylsmlib import BZIP2, GZIP, NO_ZIP, read_data_array, write_data_array


def field(dims, seed=0):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal(dims))


def test_layout_is_dims_then_x_fastest_values(tmp_path):
    a = field((5, 4, 3))
    name = write_data_array(str(tmp_path / "phi.dat"), a, grid_dims_ghostbox=(5, 4, 3))
    raw = open(name, "rb").read()
    assert np.frombuffer(raw[:12], dtype=np.intc).tolist() == [5, 4, 3]
    vals = np.frombuffer(raw[12:], dtype=np.float64)
    assert vals.size == 60
    # element (i, j, k) at i + 5 (j + 4 k)
    assert vals[2 + 5 * (1 + 4 * 2)] == a[2, 1, 2]


@pytest.mark.parametrize("zip_status,suffix", [(NO_ZIP, ""), (GZIP, ".gz"), (BZIP2, ".bz2")])
def test_round_trip(tmp_path, zip_status, suffix):
    a = field((7, 6, 5), seed=1)
    name = write_data_array(str(tmp_path / "phi.dat"), a, zip_status=zip_status)
    assert name.endswith("phi.dat" + suffix) and os.path.exists(name)
    dims, b = read_data_array(name)
    assert dims == (7, 6, 5)
    assert np.array_equal(b, a)


def test_tensor_and_fortran_array_write_the_same_bytes(tmp_path):
    a = field((6, 5, 4), seed=2)
    t = torch.from_numpy(np.ascontiguousarray(a.T))     # (nz, ny, nx)
    n1 = write_data_array(str(tmp_path / "a.dat"), a)
    n2 = write_data_array(str(tmp_path / "t.dat"), t)
    assert open(n1, "rb").read() == open(n2, "rb").read()


def test_dims_mismatch_is_rejected(tmp_path):
    with pytest.raises(ValueError):
        write_data_array(str(tmp_path / "x.dat"), field((3, 3, 3)), grid_dims_ghostbox=(3, 3, 4))


# ---- pinned against the reference's own writer and reader ----------------------

import ctypes  # noqa: E402
import importlib.util  # noqa: E402

from pylsmlib import read_data_array_1d, write_data_array_1d  # noqa: E402

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF_LIB = os.path.join(os.path.dirname(GOLDEN_DIR), "..", "oracle", "_ref",
                       "libdataarrays.so")


def golden_fields():
    """The seeded fields the reference wrote into tests/golden/data_array_*.dat."""
    spec = importlib.util.spec_from_file_location(
        "gen_data_array_golden", os.path.join(GOLDEN_DIR, "gen_data_array_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.fields()


def test_writer_matches_reference_golden_bytes(tmp_path):
    """writeDataArrayNoGrid / writeDataArray1d of the reference wrote the
    golden files; ours writes the same bytes."""
    a3, a1 = golden_fields()
    ours = write_data_array(str(tmp_path / "a3.dat"), a3)
    assert open(ours, "rb").read() == open(os.path.join(GOLDEN_DIR, "data_array_3d.dat"),
                                           "rb").read()
    ours = write_data_array_1d(str(tmp_path / "a1.dat"), a1)
    assert open(ours, "rb").read() == open(os.path.join(GOLDEN_DIR, "data_array_1d.dat"),
                                           "rb").read()


def test_reader_reads_reference_golden():
    a3, a1 = golden_fields()
    dims, b3 = read_data_array(os.path.join(GOLDEN_DIR, "data_array_3d.dat"))
    assert dims == a3.shape and np.array_equal(b3, a3)
    assert np.array_equal(read_data_array_1d(os.path.join(GOLDEN_DIR, "data_array_1d.dat")), a1)


@pytest.mark.parametrize("zip_status", [NO_ZIP, GZIP, BZIP2])
def test_1d_round_trip(tmp_path, zip_status):
    a = np.random.default_rng(3).standard_normal(29)
    name = write_data_array_1d(str(tmp_path / "v.dat"), a, zip_status=zip_status)
    assert np.array_equal(read_data_array_1d(name), a)


@pytest.fixture(scope="module")
def ref():
    """The reference's own data-array routines (oracle/_ref, built where the
    reference sources are present)."""
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libdataarrays.so not built (make -C oracle ref)")
    lib = ctypes.CDLL(REF_LIB)
    lib.readDataArray.restype = ctypes.c_void_p
    lib.readDataArray.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.writeDataArrayNoGrid.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                         ctypes.c_int]
    return lib


@pytest.mark.parametrize("zip_status", [NO_ZIP, GZIP, BZIP2])
def test_reference_reader_reads_our_files(tmp_path, ref, zip_status):
    a = field((6, 5, 4), seed=7)
    name = write_data_array(str(tmp_path / "phi.dat"), a, zip_status=zip_status)
    dims = np.zeros(3, dtype=np.intc)
    p = ref.readDataArray(dims.ctypes.data, name.encode())
    assert p
    vals = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)),
                                 shape=(a.size,)).copy()
    ctypes.CDLL(None).free(ctypes.c_void_p(p))
    assert dims.tolist() == [6, 5, 4]
    assert np.array_equal(vals.reshape((6, 5, 4), order="F"), a)


@pytest.mark.parametrize("zip_status,suffix", [(GZIP, ".gz"), (BZIP2, ".bz2")])
def test_we_read_compressed_reference_files(tmp_path, ref, zip_status, suffix):
    a = field((4, 6, 3), seed=8)
    dims = np.array(a.shape, dtype=np.intc)
    base = str(tmp_path / "phi.dat")
    ref.writeDataArrayNoGrid(a.ctypes.data, dims.ctypes.data, base.encode(), zip_status)
    got_dims, b = read_data_array(base + suffix)
    assert got_dims == a.shape and np.array_equal(b, a)
