"""Seeded synthetic inputs of the benchmark configurations.

No public data set is involved: every configuration is a level set built
from analytic shapes on a uniform grid with 3 ghost cells per side and cell
centres at x_lo + (i + 1/2) dx.  Random draws use numpy's PCG64 with the seed
recorded in each description.

* ``config1`` -- 64^3 on [-1,1]^3, sphere r = 0.25 at (0.1,-0.05,0),
  constant velocity (1, 0.5, 0.25), CFL 0.5, 100 steps.
* ``config2`` -- 256^3 on [-1,1]^3, union of 6 spheres (centres U(-0.6,0.6)^3,
  radii U(0.1,0.3)), speed F = 1 + 0.2 sin(4 pi x) sin(4 pi y) sin(4 pi z),
  CFL 0.5, 200 steps, reinitialization every 10 steps (20 pseudo-steps).
* ``config3`` -- 512^3 on [0,1]^3, sphere r = 0.15 at (0.35,0.35,0.35),
  LeVeque deformation field with period 3, run to t = 3.
* ``distance_case`` -- n^3 grid points on [-1,1]^3 (no ghost cells), the
  config-2 union of spheres scaled by 1.2 + 0.5 sin(3 pi x) sin(2 pi y)
  cos(pi z): the same zero level set, no longer a distance function; the
  input of the signed-distance (fast marching) benchmark.
"""
import numpy as np

SEED = 20261203


def axes(n, lo, hi, ghost=3):
    dx = [(hi[d] - lo[d]) / n[d] for d in range(3)]
    ax = [lo[d] + (np.arange(-ghost, n[d] + ghost) + 0.5) * dx[d] for d in range(3)]
    return ax, dx


def union_of_spheres(ax, centres, radii, dtype=np.float64):
    """min_l |x - c_l| - r_l on the grid of axes ``ax`` (Fortran order)."""
    x = ax[0][:, None, None]
    y = ax[1][None, :, None]
    z = ax[2][None, None, :]
    shape = (len(ax[0]), len(ax[1]), len(ax[2]))
    phi = np.full(shape, np.inf, dtype=np.float64, order="F")
    for c, r in zip(centres, radii):
        d = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r
        np.minimum(phi, d, out=phi)
    return np.asfortranarray(phi.astype(dtype))


def config1(n=64):
    ax, dx = axes((n, n, n), (-1, -1, -1), (1, 1, 1))
    phi = union_of_spheres(ax, [(0.1, -0.05, 0.0)], [0.25])
    vel = [np.full(phi.shape, v, order="F") for v in (1.0, 0.5, 0.25)]
    return {"n": (n, n, n), "dx": dx, "phi": phi, "vel": vel, "cfl": 0.5,
            "steps": 100}


def config2_spheres(seed=SEED):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.6, 0.6, size=(6, 3))
    radii = rng.uniform(0.1, 0.3, size=6)
    return centres, radii


def config2(n=256, seed=SEED, dtype=np.float64):
    ax, dx = axes((n, n, n), (-1, -1, -1), (1, 1, 1))
    centres, radii = config2_spheres(seed)
    phi = union_of_spheres(ax, centres, radii, dtype)
    s = [np.sin(4 * np.pi * a) for a in ax]
    F = 1.0 + 0.2 * s[0][:, None, None] * s[1][None, :, None] * s[2][None, None, :]
    F = np.asfortranarray(F.astype(dtype))
    return {"n": (n, n, n), "dx": dx, "phi": phi, "F": F, "cfl": 0.5,
            "steps": 200, "reinit_interval": 10, "reinit_iters": 20,
            "use_phi0": 0, "seed": seed, "x_lo": (-1.0, -1.0, -1.0)}


def distance_case(n=256, seed=SEED):
    """(phi, dx): phi an (n, n, n) Fortran-ordered array (x fastest) of grid
    points x_i = -1 + i dx, dx = 2/(n-1); dx in x, y, z order."""
    a = np.linspace(-1.0, 1.0, n)
    dx = [2.0 / (n - 1)] * 3
    centres, radii = config2_spheres(seed)
    phi = union_of_spheres([a, a, a], centres, radii)
    scale = (1.2 + 0.5 * np.sin(3 * np.pi * a)[:, None, None] *
             np.sin(2 * np.pi * a)[None, :, None] * np.cos(np.pi * a)[None, None, :])
    return np.asfortranarray(phi * scale), dx


def config3(n=512, dtype=np.float64):
    ax, dx = axes((n, n, n), (0, 0, 0), (1, 1, 1))
    phi = union_of_spheres(ax, [(0.35, 0.35, 0.35)], [0.15], dtype)
    return {"n": (n, n, n), "dx": dx, "phi": phi, "cfl": 0.5, "t_end": 3.0,
            "period": 3.0, "x_lo": (0.0, 0.0, 0.0)}


def boxes(n, ghost=3):
    """(gb, fb) tuples with the interior at 0..n-1."""
    gb = (-ghost, n[0] - 1 + ghost, -ghost, n[1] - 1 + ghost, -ghost, n[2] - 1 + ghost)
    fb = (0, n[0] - 1, 0, n[1] - 1, 0, n[2] - 1)
    return gb, fb


def config4(ngrids=256, seed=SEED + 4, lo_n=32, hi_n=128):
    """256 grids, per-axis sizes U{32..128}, each on [-1,1]^3 (dx = 2/n per
    axis), a union of 1-8 spheres (centres U(-0.6,0.6)^3, radii U(0.1,0.3)),
    a constant velocity U(-1,1)^3, CFL 0.5, 50 steps, periodic boundaries
    (the boundary condition of the reference's 3D advection example)."""
    rng = np.random.default_rng(seed)
    sizes, dxs, vels, grids = [], [], [], []
    for _ in range(ngrids):
        n = tuple(int(v) for v in rng.integers(lo_n, hi_n + 1, size=3))
        ax, dx = axes(n, (-1, -1, -1), (1, 1, 1))
        k = int(rng.integers(1, 9))
        centres = rng.uniform(-0.6, 0.6, size=(k, 3))
        radii = rng.uniform(0.1, 0.3, size=k)
        sizes.append(n)
        dxs.append(tuple(dx))
        vels.append(tuple(rng.uniform(-1, 1, size=3)))
        grids.append((ax, centres, radii))
    return {"sizes": sizes, "dx": dxs, "vel": vels, "grids": grids, "cfl": 0.5,
            "steps": 50, "seed": seed, "bc": "periodic"}


def config4_phi(cfg, dtype=np.float64):
    return [union_of_spheres(ax, c, r, dtype) for ax, c, r in cfg["grids"]]


def config5(n=128, lattice=8, seed=SEED + 5):
    """128^3 on [-1,1]^3; velocity a trilinear B-spline on a lattice^3
    lattice spanning the domain, coefficients N(0, 0.5^2); phi0 a sphere of
    radius 0.3 at the origin; target an ellipsoid with semi-axes
    (0.4, 0.3, 0.25), implicit function scaled by the smallest semi-axis;
    200 steps, dt frozen at the CFL 0.5 value of t = 0; Heaviside width
    1.5 dx."""
    rng = np.random.default_rng(seed)
    ax, dx = axes((n, n, n), (-1, -1, -1), (1, 1, 1))
    theta = rng.normal(0.0, 0.5, size=(3, lattice, lattice, lattice))
    phi0 = union_of_spheres(ax, [(0.0, 0.0, 0.0)], [0.3])
    x = ax[0][:, None, None]
    y = ax[1][None, :, None]
    z = ax[2][None, None, :]
    target = (np.sqrt((x / 0.4) ** 2 + (y / 0.3) ** 2 + (z / 0.25) ** 2) - 1.0) * 0.25
    return {"n": (n, n, n), "dx": dx, "x_lo": (-1.0, -1.0, -1.0), "lattice": lattice,
            "theta": theta, "phi0": phi0, "target": np.asfortranarray(target),
            "steps": 200, "cfl": 0.5, "eps": 1.5 * dx[0], "seed": seed}
