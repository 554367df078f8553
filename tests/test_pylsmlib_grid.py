"""pylsmlib.Grid reproduces the serial package's grid arithmetic
(src/serial/lsm_grid.c:46, :50-190, :788-982, lsm_initialization3d.c:55-57)."""
import pytest

from pylsmlib import Grid


@pytest.mark.parametrize("accuracy,ghost,lo_shift,hi_shift",
                         [("LOW", 2, 0, 1), ("MEDIUM", 3, 2, 2), ("HIGH", 5, 3, 4),
                          ("VERY_HIGH", 4, 2, 3)])
def test_index_spaces(accuracy, ghost, lo_shift, hi_shift):
    g = Grid.set_grid_dims((20, 12, 9), (-1.0, 0.0, 2.0), (1.0, 0.6, 2.9), accuracy)
    assert g.num_ghostcells == ghost
    assert g.grid_dims_ghostbox == (20 + 2 * ghost, 12 + 2 * ghost, 9 + 2 * ghost)
    assert g.gb == (0, 19 + 2 * ghost, 0, 11 + 2 * ghost, 0, 8 + 2 * ghost)
    # D1 fill box = ghost box shrunk by one; the scheme's fill box from it
    d1 = (1, 18 + 2 * ghost, 1, 10 + 2 * ghost, 1, 7 + 2 * ghost)
    assert g.D1_fb == d1
    assert g.fb == (1 + lo_shift, d1[1] - hi_shift, 1 + lo_shift, d1[3] - hi_shift,
                    1 + lo_shift, d1[5] - hi_shift)
    assert g.num_gridpts == (20 + 2 * ghost) * (12 + 2 * ghost) * (9 + 2 * ghost)


def test_set_dx_rounds_the_extent_and_resets_x_hi():
    g = Grid.set_dx(0.1, (0.0, 0.0, 0.0), (1.04, 0.5, 0.26))
    assert g.grid_dims == (10, 5, 3)
    assert g.x_hi == (0.0 + 10 * 0.1, 0.0 + 5 * 0.1, 0.0 + 3 * 0.1)
    assert g.x_lo_ghostbox == (-0.4, -0.4, -0.4)
    assert g.shape == (3 + 8, 5 + 8, 10 + 8)


def test_grid_point_coordinates():
    g = Grid.set_dx((0.1, 0.2, 0.25), (0.0, -1.0, 2.0), (1.0, 1.0, 3.0))
    x, y, z = g.coordinates(device="cpu")
    assert x.shape == g.shape
    assert float(x[0, 0, 0]) == g.x_lo_ghostbox[0]
    assert float(x[0, 0, 5]) == g.x_lo_ghostbox[0] + 0.1 * 5
    assert float(y[0, 3, 0]) == g.x_lo_ghostbox[1] + 0.2 * 3
    assert float(z[2, 0, 0]) == g.x_lo_ghostbox[2] + 0.25 * 2


# ---- pinned against the reference's own grid constructors ------------------------

import ctypes  # noqa: E402
import importlib.util  # noqa: E402
import json  # noqa: E402
import os  # noqa: E402

import numpy as np  # noqa: E402

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def ours(ctor, arg, x_lo, x_hi, accuracy):
    if ctor == "set_grid_dims":
        return Grid.set_grid_dims(arg, x_lo, x_hi, accuracy)
    return Grid.set_dx(arg, x_lo, x_hi, accuracy)


def as_fields(g):
    return {"num_dims": g.num_dims, "x_lo": list(g.x_lo), "x_hi": list(g.x_hi),
            "x_lo_ghostbox": list(g.x_lo_ghostbox), "x_hi_ghostbox": list(g.x_hi_ghostbox),
            "grid_dims": list(g.grid_dims), "grid_dims_ghostbox": list(g.grid_dims_ghostbox),
            "dx": list(g.dx), "num_gridpts": g.num_gridpts, "gb": list(g.gb),
            "fb": list(g.fb), "D1_fb": list(g.D1_fb), "D2_fb": list(g.D2_fb),
            "D3_fb": list(g.D3_fb), "num_nb_levels": g.num_nb_levels,
            "marks": [g.mark_gb, g.mark_D1, g.mark_D2, g.mark_D3, g.mark_fb],
            "beta": g.beta, "gamma": g.gamma}


GOLDEN = json.load(open(os.path.join(GOLDEN_DIR, "grid_golden.json")))


@pytest.mark.parametrize("case", GOLDEN, ids=["%s-%s-%d" % (c["ctor"], c["accuracy"], i)
                                              for i, c in enumerate(GOLDEN)])
def test_grid_matches_reference_golden(case):
    """Every field of the reference's Grid, as createGridSetDx /
    createGridSetDxDyDz / createGridSetGridDims filled it, is ours exactly."""
    g = ours(case["ctor"], case["arg"], case["x_lo"], case["x_hi"], case["accuracy"])
    assert as_fields(g) == case["grid"]


def test_grid_matches_reference_live_on_seeded_extents():
    """Where the reference's grid code is built (oracle/_ref/libgrid.so),
    seeded spacings and extents agree field by field."""
    lib_path = os.path.join(os.path.dirname(GOLDEN_DIR), "..", "oracle", "_ref", "libgrid.so")
    if not os.path.exists(lib_path):
        pytest.skip("oracle/_ref/libgrid.so not built (make -C oracle ref)")
    spec = importlib.util.spec_from_file_location(
        "gen_grid_golden", os.path.join(GOLDEN_DIR, "gen_grid_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    lib = ctypes.CDLL(lib_path)
    lib.createGridSetDxDyDz.restype = ctypes.POINTER(gen.RefGrid)
    lib.createGridSetDxDyDz.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [
        gen.D3, gen.D3, ctypes.c_int]
    lib.createGridSetGridDims.restype = ctypes.POINTER(gen.RefGrid)
    lib.createGridSetGridDims.argtypes = [ctypes.c_int, gen.I3, gen.D3, gen.D3, ctypes.c_int]
    lib.destroyGrid.argtypes = [ctypes.POINTER(gen.RefGrid)]
    rng = np.random.default_rng(11)
    for _ in range(40):
        lo = rng.uniform(-2, 1, 3)
        hi = lo + rng.uniform(0.1, 3, 3)
        h = rng.uniform(0.005, 0.2, 3)
        dims = rng.integers(1, 90, 3)
        acc = int(rng.integers(0, 4))
        p = lib.createGridSetDxDyDz(3, *h, gen.D3(*lo), gen.D3(*hi), acc)
        assert gen.fields(p.contents) == as_fields(
            Grid.set_dx(tuple(h), tuple(lo), tuple(hi), gen.ACCURACY[acc]))
        lib.destroyGrid(p)
        p = lib.createGridSetGridDims(3, gen.I3(*dims), gen.D3(*lo), gen.D3(*hi), acc)
        assert gen.fields(p.contents) == as_fields(
            Grid.set_grid_dims(tuple(int(v) for v in dims), tuple(lo), tuple(hi),
                               gen.ACCURACY[acc]))
        lib.destroyGrid(p)


# ---- binary grid files (lsm_grid.c:613-787) ---------------------------------------

def _golden_binary_case():
    case = [c for c in GOLDEN if c["ctor"] == "set_dxdydz"][4]   # the second such case
    return case["arg"], case["x_lo"], case["x_hi"]


@pytest.mark.parametrize("accuracy,name", [("VERY_HIGH", "very_high"), ("HIGH", "high")])
def test_binary_grid_file_matches_reference_writer(tmp_path, accuracy, name):
    """writeGridToBinaryFile of the reference wrote the golden files; ours
    writes the same bytes and reads them back field by field."""
    h, lo, hi = _golden_binary_case()
    g = Grid.set_dx(tuple(h), tuple(lo), tuple(hi), accuracy)
    golden = os.path.join(GOLDEN_DIR, "grid_%s.bin" % name)
    ours = g.write_binary(str(tmp_path / "grid.bin"))
    assert open(ours, "rb").read() == open(golden, "rb").read()
    back = Grid.read_binary(golden)
    assert as_fields(back) == as_fields(g) and back.accuracy == accuracy


@pytest.mark.parametrize("zip_status,suffix", [(0, ""), (1, ".gz"), (2, ".bz2")])
def test_reference_reads_our_binary_grid_files(tmp_path, zip_status, suffix):
    lib_path = os.path.join(os.path.dirname(GOLDEN_DIR), "..", "oracle", "_ref", "libgrid.so")
    if not os.path.exists(lib_path):
        pytest.skip("oracle/_ref/libgrid.so not built (make -C oracle ref)")
    spec = importlib.util.spec_from_file_location(
        "gen_grid_golden", os.path.join(GOLDEN_DIR, "gen_grid_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    lib = ctypes.CDLL(lib_path)
    lib.readGridFromBinaryFile.restype = ctypes.POINTER(gen.RefGrid)
    lib.readGridFromBinaryFile.argtypes = [ctypes.c_char_p]
    lib.destroyGrid.argtypes = [ctypes.POINTER(gen.RefGrid)]
    g = Grid.set_grid_dims((21, 17, 9), (-1.0, 0.0, 0.5), (1.0, 0.8, 1.4), "MEDIUM")
    name = g.write_binary(str(tmp_path / "grid.bin"), zip_status=zip_status)
    assert name.endswith("grid.bin" + suffix)
    p = lib.readGridFromBinaryFile(name.encode())
    assert gen.fields(p.contents) == as_fields(g)
    lib.destroyGrid(p)


def test_ascii_grid_file_matches_reference_writer(tmp_path):
    """writeGridToAsciiFile (printGrid) of the reference wrote the golden
    text; ours writes the same bytes."""
    h, lo, hi = _golden_binary_case()
    g = Grid.set_dx(tuple(h), tuple(lo), tuple(hi), "VERY_HIGH")
    ours = g.write_ascii(str(tmp_path / "grid.txt"))
    assert open(ours, "rb").read() == open(os.path.join(GOLDEN_DIR, "grid_very_high.txt"),
                                           "rb").read()


def test_ascii_grid_description_matches_reference_live(tmp_path):
    """Every golden grid printed by the reference's printGrid and by ours."""
    lib_path = os.path.join(os.path.dirname(GOLDEN_DIR), "..", "oracle", "_ref", "libgrid.so")
    if not os.path.exists(lib_path):
        pytest.skip("oracle/_ref/libgrid.so not built (make -C oracle ref)")
    spec = importlib.util.spec_from_file_location(
        "gen_grid_golden", os.path.join(GOLDEN_DIR, "gen_grid_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    lib = ctypes.CDLL(lib_path)
    for f in ("createGridSetDx", "createGridSetDxDyDz", "createGridSetGridDims"):
        getattr(lib, f).restype = ctypes.POINTER(gen.RefGrid)
    lib.createGridSetDx.argtypes = [ctypes.c_int, ctypes.c_double, gen.D3, gen.D3, ctypes.c_int]
    lib.createGridSetDxDyDz.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [
        gen.D3, gen.D3, ctypes.c_int]
    lib.createGridSetGridDims.argtypes = [ctypes.c_int, gen.I3, gen.D3, gen.D3, ctypes.c_int]
    lib.writeGridToAsciiFile.argtypes = [ctypes.POINTER(gen.RefGrid), ctypes.c_char_p,
                                         ctypes.c_int]
    lib.destroyGrid.argtypes = [ctypes.POINTER(gen.RefGrid)]
    name = str(tmp_path / "ref.txt")
    for case in GOLDEN:
        acc = gen.ACCURACY.index(case["accuracy"])
        lo, hi, arg = gen.D3(*case["x_lo"]), gen.D3(*case["x_hi"]), case["arg"]
        if case["ctor"] == "set_dx":
            p = lib.createGridSetDx(3, arg, lo, hi, acc)
        elif case["ctor"] == "set_dxdydz":
            p = lib.createGridSetDxDyDz(3, *arg, lo, hi, acc)
        else:
            p = lib.createGridSetGridDims(3, gen.I3(*arg), lo, hi, acc)
        lib.writeGridToAsciiFile(p, name.encode(), 0)
        lib.destroyGrid(p)
        g = ours(case["ctor"], case["arg"], case["x_lo"], case["x_hi"], case["accuracy"])
        assert open(name).read() == g.describe(), case
