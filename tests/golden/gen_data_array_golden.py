"""Writes the data-array golden files with the reference's own writer.

The reference's writeDataArrayNoGrid and writeDataArray1d
(src/serial/lsm_data_arrays.c:380-397, :439-454) come from
oracle/_ref/libdataarrays.so, built by `make -C oracle ref` from the
reference sources. The fields are seeded. Run from the repository root:

    python tests/golden/gen_data_array_golden.py
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "..", "oracle", "_ref", "libdataarrays.so")


def fields():
    """The 3D field (dims (5, 4, 3), Fortran order) and the 1D field."""
    rng = np.random.default_rng(20261203)
    return (np.asfortranarray(rng.standard_normal((5, 4, 3))),
            rng.standard_normal(17))


def main():
    lib = ctypes.CDLL(LIB)
    a3, a1 = fields()
    dims = np.array(a3.shape, dtype=np.intc)
    lib.writeDataArrayNoGrid(a3.ctypes.data_as(ctypes.c_void_p),
                             dims.ctypes.data_as(ctypes.c_void_p),
                             os.path.join(HERE, "data_array_3d.dat").encode(), 0)
    lib.writeDataArray1d(a1.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(a1.size),
                         os.path.join(HERE, "data_array_1d.dat").encode(), 0)


if __name__ == "__main__":
    main()
