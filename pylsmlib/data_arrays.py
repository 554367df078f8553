"""The serial package's data-array file format (src/serial/lsm_data_arrays.c).

A file holds three native ints -- the ghost-box dimensions nx, ny, nz -- and
then nx*ny*nz LSMLIB_REAL values with x fastest (writeDataArray, :363-377;
writeDataArrayNoGrid, :380-397; readDataArray, :400-435).  With zip status
GZIP or BZIP2 the written file is compressed in place to name.gz / name.bz2,
and a name ending in .gz / .bz2 is decompressed before reading
(lsm_file.c:18-90).  Fields may be CUDA tensors (shape (nz, ny, nx), the
layout of the reference's arrays), host tensors or numpy arrays.
"""
import bz2
import gzip
import os

import numpy as np

NO_ZIP, GZIP, BZIP2 = 0, 1, 2


def _host_xyz(data):
    """(array in x-fastest memory order, (nx, ny, nz))."""
    try:
        import torch
        if isinstance(data, torch.Tensor):
            a = data.detach().contiguous().cpu().numpy()      # (nz, ny, nx), C order
            return a, tuple(reversed(a.shape))
    except ImportError:
        pass
    a = np.asarray(data)
    if a.flags.f_contiguous and not a.flags.c_contiguous:
        return a, a.shape                                     # (nx, ny, nz), Fortran
    return np.ascontiguousarray(a), tuple(reversed(a.shape))  # treated as (nz, ny, nx)


def write_data_array(file_name, data, grid_dims_ghostbox=None, zip_status=NO_ZIP,
                     dtype=np.float64):
    """writeDataArray / writeDataArrayNoGrid: the dims, then the values
    (``dtype``: the library's LSMLIB_REAL).  Returns the name written."""
    a, dims = _host_xyz(data)
    if grid_dims_ghostbox is not None and tuple(grid_dims_ghostbox) != tuple(dims):
        raise ValueError("data has dims %s, grid says %s" % (dims, tuple(grid_dims_ghostbox)))
    payload = (np.asarray(dims, dtype=np.intc).tobytes() +
               np.asarray(a, dtype=dtype).tobytes(order="A"))
    return _write(file_name, payload, zip_status)


def _write(file_name, payload, zip_status):
    """The file, compressed in place to name.gz / name.bz2 by zip status
    (zipFile, lsm_file.c:55-90); returns the name written."""
    if zip_status == GZIP:
        file_name = file_name + ".gz"
        with gzip.open(file_name, "wb") as f:
            f.write(payload)
    elif zip_status == BZIP2:
        file_name = file_name + ".bz2"
        with bz2.open(file_name, "wb") as f:
            f.write(payload)
    else:
        with open(file_name, "wb") as f:
            f.write(payload)
    return file_name


def _read(file_name):
    """The file's bytes, through the decompressor its name asks for
    (checkUnzipFile, lsm_file.c:18-53)."""
    if file_name.endswith(".gz"):
        opener = gzip.open
    elif file_name.endswith(".bz2"):
        opener = bz2.open
    else:
        opener = open
    if not os.path.exists(file_name):
        raise FileNotFoundError(file_name)
    with opener(file_name, "rb") as f:
        return f.read()


def read_data_array(file_name, dtype=np.float64):
    """readDataArray: (grid_dims_ghostbox, array of shape (nx, ny, nz) in
    Fortran order).  Compressed names are read through the decompressor."""
    raw = _read(file_name)
    head = np.dtype(np.intc).itemsize * 3
    dims = tuple(int(v) for v in np.frombuffer(raw[:head], dtype=np.intc))
    n = dims[0] * dims[1] * dims[2]
    vals = np.frombuffer(raw[head:head + n * np.dtype(dtype).itemsize], dtype=dtype)
    if vals.size != n:
        raise ValueError("%s: %d values for dims %s" % (file_name, vals.size, dims))
    return dims, vals.reshape(dims, order="F").copy(order="F")


def write_data_array_1d(file_name, data, zip_status=NO_ZIP, dtype=np.float64):
    """writeDataArray1d (lsm_data_arrays.c:439-454): the number of elements
    as one native int, then the values.  Returns the name written."""
    a = np.asarray(data, dtype=dtype).ravel()
    payload = np.asarray([a.size], dtype=np.intc).tobytes() + a.tobytes()
    return _write(file_name, payload, zip_status)


def read_data_array_1d(file_name, dtype=np.float64):
    """readDataArray1d (lsm_data_arrays.c:457-489): the values as a 1D
    array."""
    raw = _read(file_name)
    head = np.dtype(np.intc).itemsize
    n = int(np.frombuffer(raw[:head], dtype=np.intc)[0])
    vals = np.frombuffer(raw[head:head + n * np.dtype(dtype).itemsize], dtype=dtype)
    if vals.size != n:
        raise ValueError("%s: %d values for %d elements" % (file_name, vals.size, n))
    return vals.copy()
