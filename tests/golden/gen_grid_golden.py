"""Writes tests/golden/grid_golden.json with the reference's own grid
constructors, grid_{very_high,high}.bin with its binary grid writer and
grid_very_high.txt with its ASCII grid writer.

createGridSetDx, createGridSetDxDyDz and createGridSetGridDims
(src/serial/lsm_grid.c:50-250, with setIndexSpaceLimits* at :788-1040) and
writeGridToBinaryFile (:613-676) come
from oracle/_ref/libgrid.so, built by `make -C oracle ref` from the reference
sources. Run from the repository root:

    python tests/golden/gen_grid_golden.py
"""
import ctypes
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "..", "..", "oracle", "_ref", "libgrid.so")
ACCURACY = ["LOW", "MEDIUM", "HIGH", "VERY_HIGH"]   # LSMLIB_SPATIAL_DERIVATIVE_ACCURACY_TYPE
D3 = ctypes.c_double * 3
I3 = ctypes.c_int * 3


class RefGrid(ctypes.Structure):
    """struct _Grid of the FP64 build (lsm_grid.h:43-95)."""
    _fields_ = ([("num_dims", ctypes.c_int)] +
                [(n, D3) for n in ("x_lo", "x_hi", "x_lo_ghostbox", "x_hi_ghostbox")] +
                [("grid_dims", I3), ("grid_dims_ghostbox", I3), ("dx", D3),
                 ("num_gridpts", ctypes.c_int)] +
                [(a + b + "_" + box, ctypes.c_int) for box in ("gb", "fb", "D1_fb", "D2_fb",
                                                                "D3_fb")
                 for a in "ijk" for b in ("lo", "hi")] +
                [("num_nb_levels", ctypes.c_int)] +
                [(n, ctypes.c_ubyte) for n in ("mark_gb", "mark_D1", "mark_D2", "mark_D3",
                                               "mark_fb")] +
                [("beta", ctypes.c_double), ("gamma", ctypes.c_double)])


# (constructor, spacing or grid dims, x_lo, x_hi); the extents include ones
# that rint rounds down (10.4), up (2.6) and to even (2.5)
CASES = [
    ("set_dx", 0.1, (0.0, 0.0, 0.0), (1.04, 0.5, 0.26)),
    ("set_dx", 0.2, (-1.0, -0.5, 0.0), (1.0, 0.5, 0.5)),
    ("set_dxdydz", (0.1, 0.2, 0.25), (0.0, -1.0, 2.0), (1.0, 1.0, 3.0)),
    ("set_dxdydz", (2.0 / 64, 2.0 / 48, 2.0 / 40), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)),
    ("set_grid_dims", (20, 12, 9), (-1.0, 0.0, 2.0), (1.0, 0.6, 2.9)),
    ("set_grid_dims", (64, 64, 64), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)),
]


def fields(g):
    box = lambda name: [getattr(g, a + b + "_" + name) for a in "ijk" for b in ("lo", "hi")]
    return {"num_dims": g.num_dims, "x_lo": list(g.x_lo), "x_hi": list(g.x_hi),
            "x_lo_ghostbox": list(g.x_lo_ghostbox), "x_hi_ghostbox": list(g.x_hi_ghostbox),
            "grid_dims": list(g.grid_dims), "grid_dims_ghostbox": list(g.grid_dims_ghostbox),
            "dx": list(g.dx), "num_gridpts": g.num_gridpts, "gb": box("gb"), "fb": box("fb"),
            "D1_fb": box("D1_fb"), "D2_fb": box("D2_fb"), "D3_fb": box("D3_fb"),
            "num_nb_levels": g.num_nb_levels,
            "marks": [g.mark_gb, g.mark_D1, g.mark_D2, g.mark_D3, g.mark_fb],
            "beta": g.beta, "gamma": g.gamma}


def main():
    lib = ctypes.CDLL(LIB)
    for f in ("createGridSetDx", "createGridSetDxDyDz", "createGridSetGridDims"):
        getattr(lib, f).restype = ctypes.POINTER(RefGrid)
    lib.createGridSetDx.argtypes = [ctypes.c_int, ctypes.c_double, D3, D3, ctypes.c_int]
    lib.createGridSetDxDyDz.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [D3, D3,
                                                                                   ctypes.c_int]
    lib.createGridSetGridDims.argtypes = [ctypes.c_int, I3, D3, D3, ctypes.c_int]
    lib.destroyGrid.argtypes = [ctypes.POINTER(RefGrid)]
    out = []
    for ctor, h, lo, hi in CASES:
        for acc, name in enumerate(ACCURACY):
            if ctor == "set_dx":
                p = lib.createGridSetDx(3, h, D3(*lo), D3(*hi), acc)
            elif ctor == "set_dxdydz":
                p = lib.createGridSetDxDyDz(3, *h, D3(*lo), D3(*hi), acc)
            else:
                p = lib.createGridSetGridDims(3, I3(*h), D3(*lo), D3(*hi), acc)
            out.append({"ctor": ctor, "arg": h, "x_lo": lo, "x_hi": hi, "accuracy": name,
                        "grid": fields(p.contents)})
            lib.destroyGrid(p)
    with open(os.path.join(HERE, "grid_golden.json"), "w") as f:
        json.dump(out, f, indent=0)
    # binary grid files: the second set_dxdydz case at two accuracies
    lib.writeGridToBinaryFile.argtypes = [ctypes.POINTER(RefGrid), ctypes.c_char_p,
                                          ctypes.c_int]
    _, h, lo, hi = CASES[3]
    lib.writeGridToAsciiFile.argtypes = [ctypes.POINTER(RefGrid), ctypes.c_char_p,
                                         ctypes.c_int]
    for acc, name in ((3, "very_high"), (2, "high")):
        p = lib.createGridSetDxDyDz(3, *h, D3(*lo), D3(*hi), acc)
        lib.writeGridToBinaryFile(p, os.path.join(HERE, "grid_%s.bin" % name).encode(), 0)
        if name == "very_high":
            lib.writeGridToAsciiFile(p, os.path.join(HERE, "grid_%s.txt" % name).encode(), 0)
        lib.destroyGrid(p)


if __name__ == "__main__":
    main()
