"""Seeded input cases for the toolbox golden fixtures.

Two cases per routine, both on a grid whose fill box has odd extents and
non-zero lower bounds:

* ``smooth`` -- sphere signed distance plus a small perturbation;
* ``degenerate`` -- values quantised to multiples of 1/8 (ties in every ENO
  comparison), a flat region (all WENO differences zero), velocities that are
  exactly zero, below the zero tolerance (1e-13) and of both signs.
"""
import numpy as np

from lsmlib_b200 import abi
from lsmlib_b200.toolbox import Field

FB_LO = (-2, 3, 1)
FB_N = (6, 5, 4)
GHOST = 3


def boxes():
    fb = (FB_LO[0], FB_LO[0] + FB_N[0] - 1, FB_LO[1], FB_LO[1] + FB_N[1] - 1,
          FB_LO[2], FB_LO[2] + FB_N[2] - 1)
    glo = tuple(l - GHOST for l in FB_LO)
    ghi = tuple(l + n - 1 + GHOST for l, n in zip(FB_LO, FB_N))
    return fb, glo, ghi


def make_inputs(sym, case, seed):
    """Arrays and scalars for routine ``sym``; returns (fields, scalars, fb)."""
    rng = np.random.default_rng(seed)
    fb, glo, ghi = boxes()
    shape = tuple(h - l + 1 for l, h in zip(glo, ghi))
    idx = np.meshgrid(*[np.arange(l, h + 1) for l, h in zip(glo, ghi)], indexing="ij")
    h = 0.13

    def level_set():
        x, y, z = (i * h for i in idx)
        r = np.sqrt((x - 0.05) ** 2 + (y - 0.55) ** 2 + (z - 0.4) ** 2)
        phi = r - 0.45
        if case == "smooth":
            return phi + 1e-3 * rng.standard_normal(shape)
        q = np.round(phi * 8.0) / 8.0
        q[: shape[0] // 2, : shape[1] // 2, :] = 0.25      # flat block
        return q

    def velocity():
        if case == "smooth":
            return rng.standard_normal(shape)
        v = rng.choice([-1.0, -0.5, 0.0, 1e-13, -1e-13, 0.5, 1.0], size=shape)
        return v

    def generic():
        if case == "smooth":
            return rng.standard_normal(shape)
        return np.round(rng.standard_normal(shape) * 4.0) / 4.0

    fields, scalars = {}, {}
    for kind, name in abi.parse(abi.SIGNATURES[sym]):
        if kind in ("I", "X", "O"):
            if name in ("phi", "phi0", "S", "u_cur", "u_stage1", "u_stage2", "field1"):
                data = level_set()
                if name in ("phi0", "u_stage1", "u_stage2", "S"):
                    data = data + (0.01 * rng.standard_normal(shape) if case == "smooth"
                                   else np.round(rng.standard_normal(shape)) / 16.0)
            elif name == "field2":
                data = level_set() + (rng.standard_normal(shape) * 1e-3)
            elif name.startswith("vel") or name.startswith("signed_normal"):
                data = velocity()
            elif name == "distance0":
                # the subcell-fix flag -1000 max(dx) in about half the cells
                data = np.where(rng.random(shape) < 0.5, -1000.0 * 0.17, generic())
            elif name == "psi":
                data = level_set()[::-1, :, :] + 0.1
            else:
                data = generic()
            # float32-representable inputs keep the fixture small; the
            # arithmetic on them is still full FP64
            data = data.astype(np.float32).astype(np.float64)
            fields[name] = Field(np.asfortranarray(data), glo)
        elif kind == "R":
            scalars[name] = {"dx": 0.13, "dy": 0.11, "dz": 0.17, "dt": 0.021,
                             "cfl_number": 0.5, "b": 0.37}.get(name)
            if name == "vel_n":
                scalars[name] = 0.7 if case == "smooth" else -1.25
        elif kind == "N":
            scalars[name] = 0
    return fields, scalars, fb


# routines that write beyond the fill box: the zeroing of the whole ghost box,
# and the two RHS terms whose loops run k over [klo_fb, khi_gb], j over
# [jlo_fb, jhi_gb] and i over [ilo_gb, ihi_gb] of the RHS array
# (lsm_level_set_evolution3d.f.in:505-507, :586-588)
WHOLE_ARRAY_OUTPUT = ("lsm3dzerooutlevelseteqnrhs_",
                      "lsm3daddconstprecomputedcurvtermtolserhs_",
                      "lsm3daddexternalandnormalveltermtolserhs_")


def run(tb, sym, fields, scalars, fb):
    """Run ``sym`` on copies of ``fields``; returns {name: array or float}.

    Array outputs are the fill-box slices (the whole array for boundary
    conditions, whose ghost cells are the output)."""
    fs = {k: v.copy() for k, v in fields.items()}
    s = dict(scalars)
    out = {}
    if "bdry_location_idx" in s:
        for face in range(6):          # all faces in order, as the serial
            s["bdry_location_idx"] = face   # driver's case 9 does
            tb.call(sym, fs, fb, **s)
        out["phi"] = fs["phi"].data.copy()
        return out
    res = tb.call(sym, fs, fb, **s)
    for kind, name in abi.parse(abi.SIGNATURES[sym]):
        if kind in ("O", "X"):
            lo, hi = (fb[0], fb[2], fb[4]), (fb[1], fb[3], fb[5])
            if sym in WHOLE_ARRAY_OUTPUT:
                out[name] = fs[name].data.copy()
            else:
                out[name] = fs[name].view(lo, hi).copy()
    out.update(res)
    return out


VARIANTS = {
    # extra scalar settings exercised beyond the defaults
    "lsm3dcomputereinitializationeqnrhs_": [{"use_phi0_for_sgn": 0},
                                            {"use_phi0_for_sgn": 1}],
}
