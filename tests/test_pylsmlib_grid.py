"""pylsmlib.Grid reproduces the serial package's grid arithmetic
(src/serial/lsm_grid.c:46, :50-190, :788-982, lsm_initialization3d.c:55-57)."""
import pytest

from pylsmlib import Grid


@pytest.mark.parametrize("accuracy,ghost,lo_shift,hi_shift",
                         [("LOW", 2, 0, 1), ("MEDIUM", 3, 1, 2), ("HIGH", 5, 2, 3),
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
