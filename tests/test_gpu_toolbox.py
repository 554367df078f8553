"""GPU parity of every reference-compatible routine (C ABI, FP64, strict).

Each routine is called through liblsmgpu.so exactly as a reference caller
would call the Fortran symbol, and compared bit for bit with
* the golden outputs of the reference's own routines (tests/golden), for host
  arrays (staged path) and device arrays (in-place path);
* the C oracle on larger seeded grids."""
import numpy as np
import pytest

from cases import WHOLE_ARRAY_OUTPUT, run
from golden_util import assert_bitwise, load_cases
from lsmlib_b200 import abi
from lsmlib_b200.toolbox import Field

pytestmark = pytest.mark.gpu
CASES = load_cases()


@pytest.mark.parametrize("key,sym,fields,scalars,fb,want", CASES,
                         ids=[c[0] for c in CASES])
def test_host_arrays_match_reference_golden(gpu_tb, key, sym, fields, scalars,
                                            fb, want):
    got = run(gpu_tb, sym, fields, scalars, fb)
    assert_bitwise(got, want, key)


def run_on_device(tb, sym, fields, scalars, fb):
    from lsmlib_b200 import gpu
    dev = {k: gpu.device_field(v) for k, v in fields.items()}
    s = dict(scalars)
    out = {}
    if "bdry_location_idx" in s:
        for face in range(6):
            s["bdry_location_idx"] = face
            tb.call(sym, dev, fb, **s)
        out["phi"] = dev["phi"].data.download()
        return out
    res = tb.call(sym, dev, fb, **s)
    for kind, name in abi.parse(abi.SIGNATURES[sym]):
        if kind in ("O", "X"):
            h = gpu.host_field(dev[name])
            if sym in WHOLE_ARRAY_OUTPUT:
                out[name] = h.data
            else:
                out[name] = h.view((fb[0], fb[2], fb[4]), (fb[1], fb[3], fb[5])).copy()
    out.update(res)
    return out


@pytest.mark.parametrize("key,sym,fields,scalars,fb,want", CASES,
                         ids=[c[0] for c in CASES])
def test_device_arrays_match_reference_golden(gpu_tb, key, sym, fields, scalars,
                                              fb, want):
    got = run_on_device(gpu_tb, sym, fields, scalars, fb)
    assert_bitwise(got, want, key)


def random_case(sym, n, seed, lo=(0, 0, 0), ghost=3):
    rng = np.random.default_rng(seed)
    glo = tuple(l - ghost for l in lo)
    ghi = tuple(l + m - 1 + ghost for l, m in zip(lo, n))
    fb = (lo[0], lo[0] + n[0] - 1, lo[1], lo[1] + n[1] - 1, lo[2], lo[2] + n[2] - 1)
    shape = tuple(h - l + 1 for l, h in zip(glo, ghi))
    x = np.meshgrid(*[np.linspace(-1, 1, s) for s in shape], indexing="ij")
    sdf = np.sqrt((x[0] - 0.1) ** 2 + (x[1] + 0.05) ** 2 + x[2] ** 2) - 0.5
    fields, scalars = {}, {}
    flag = -1000.0 * max(2.0 / n[0], 2.0 / n[1], 2.0 / n[2])   # subcell-fix flag
    for kind, name in abi.parse(abi.SIGNATURES[sym]):
        if kind in "IOX":
            if name.startswith("vel") or name.startswith("signed_normal"):
                d = rng.standard_normal(shape)
            elif name == "distance0":
                d = np.where(rng.random(shape) < 0.5, flag, rng.standard_normal(shape))
            elif name.startswith("phi_") or name.startswith("S_"):
                d = rng.standard_normal(shape)
            else:
                d = sdf + 0.01 * rng.standard_normal(shape)
            fields[name] = Field(np.asfortranarray(d), glo)
        elif kind == "R":
            scalars[name] = {"dx": 2.0 / n[0], "dy": 2.0 / n[1], "dz": 2.0 / n[2],
                             "dt": 0.01, "cfl_number": 0.5, "vel_n": 0.8,
                             "b": 0.37}[name]
        elif kind == "N":
            scalars[name] = 0
    return fields, scalars, fb


@pytest.mark.parametrize("sym", sorted(abi.SIGNATURES))
@pytest.mark.parametrize("n", [(40, 30, 10), (33, 17, 9)])
def test_larger_grids_match_oracle(orc, gpu_tb, sym, n):
    fields, scalars, fb = random_case(sym, n, seed=hash((sym, n)) % 1000,
                                      lo=(-4, 2, 5))
    want = run(orc, sym, fields, scalars, fb)
    got = run(gpu_tb, sym, fields, scalars, fb)
    assert_bitwise(got, want, sym)


def test_invalid_box_is_rejected_without_writing(gpu_tb):
    from lsmlib_b200 import gpu
    fields, scalars, fb = random_case("lsm3dhjweno5_", (8, 8, 8), seed=1)
    before = fields["phi_x_plus"].data.copy()
    bad_fb = (fb[0] - 1, fb[1], fb[2], fb[3], fb[4], fb[5])  # needs 4 ghosts
    with pytest.raises(gpu.LsmgpuError) as ei:
        gpu_tb.call("lsm3dhjweno5_", fields, bad_fb, **scalars)
    assert ei.value.code == 1
    np.testing.assert_array_equal(fields["phi_x_plus"].data, before)
    # the next valid call succeeds and clears the error
    gpu_tb.call("lsm3dhjweno5_", fields, fb, **scalars)
    assert gpu.load().lsmgpu_peek_last_error() == 0


def test_empty_fill_box_is_a_no_op(gpu_tb):
    fields, scalars, fb = random_case("lsm3drk1step_", (6, 6, 6), seed=2)
    before = fields["u_next"].data.copy()
    empty = (fb[0], fb[0] - 1, fb[2], fb[3], fb[4], fb[5])
    gpu_tb.call("lsm3drk1step_", fields, empty, **scalars)
    np.testing.assert_array_equal(fields["u_next"].data, before)
