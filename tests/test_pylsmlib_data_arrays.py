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
