"""The property the reference's own boundary-condition examples print
(examples/toolbox/boundary_conditions/neumann_bc_{ENO1,ENO2,ENO3,WENO5}_3d.c):
after a homogeneous Neumann fill of all six faces, the one-sided
derivatives normal to each face vanish at the boundary cells.  The examples
print the six errors without a threshold; ENO1-3 give exactly 0, WENO5
about 5e-12 (its nonlinear weights see the mirrored stencil), so the checks
are == 0 and <= 1e-10."""
import numpy as np

from lsmlib_b200.toolbox import Field

GHOSTS = {"eno1": 1, "eno2": 2, "eno3": 3, "weno5": 3}
LIMIT = {"eno1": 0.0, "eno2": 0.0, "eno3": 0.0, "weno5": 1e-10}


def boundary_errors(call, scheme, to_device=None, to_host=None):
    """The examples' six errors (x lower/upper, y, z) for ``scheme``:
    a 40 x 30 x 10 box with the examples' quadratic phi and spacing."""
    g = GHOSTS[scheme]
    n = (40, 30, 10)
    lo, hi = (-g, -g, -g), tuple(m - 1 + g for m in n)
    shape = tuple(h - l + 1 for l, h in zip(lo, hi))
    dx, dy, dz = 1.0 / n[0], 1.0 / n[1], 1.0 / n[2]
    phi = np.zeros(shape, order="F")
    i, j, k = np.meshgrid(*[np.arange(m) for m in n], indexing="ij")
    x, y, z = (i + 0.5) * dx, (j + 0.5) * dy, (k + 0.5) * dz
    phi[g:g + n[0], g:g + n[1], g:g + n[2]] = ((x - 0.33) ** 2 + 4 * (y - 0.54) ** 2
                                               + 0.25 * (z - 0.94) ** 2 - 0.25)
    names = ("phi_x_plus", "phi_y_plus", "phi_z_plus", "phi_x_minus", "phi_y_minus",
             "phi_z_minus")
    f = {"phi": Field(np.asfortranarray(phi), lo)}
    f.update({nm: Field.zeros(lo, hi) for nm in names})
    if to_device:
        f = {k_: to_device(v) for k_, v in f.items()}
    fb = (0, n[0] - 1, 0, n[1] - 1, 0, n[2] - 1)
    for face in range(6):
        call("lsm3dhomogeneousneumann%s_" % scheme, {"phi": f["phi"]}, fb,
             bdry_location_idx=face)
    call("lsm3dhj%s_" % scheme, f, fb, dx=dx, dy=dy, dz=dz)
    if to_host:
        f = {k_: to_host(v) for k_, v in f.items()}

    def inner(nm):
        return f[nm].data[g:g + n[0], g:g + n[1], g:g + n[2]]
    return [np.abs(inner("phi_x_minus")[0]).max(), np.abs(inner("phi_x_plus")[-1]).max(),
            np.abs(inner("phi_y_minus")[:, 0]).max(), np.abs(inner("phi_y_plus")[:, -1]).max(),
            np.abs(inner("phi_z_minus")[:, :, 0]).max(),
            np.abs(inner("phi_z_plus")[:, :, -1]).max()]
