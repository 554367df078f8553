"""The C oracle reproduces the reference's own outputs bit for bit.

The golden fixture was produced by the reference's Fortran routines (built
from the reference sources by oracle/f77toc.py, see tests/golden/gen_golden.py)
on seeded smooth and degenerate inputs (ties, flat regions, zero and
sub-tolerance velocities)."""
import pytest

from cases import run
from golden_util import assert_bitwise, load_cases

CASES = load_cases()


@pytest.mark.parametrize("key,sym,fields,scalars,fb,want", CASES,
                         ids=[c[0] for c in CASES])
def test_oracle_matches_reference_golden(orc, key, sym, fields, scalars, fb, want):
    got = run(orc, sym, fields, scalars, fb)
    assert_bitwise(got, want, key)


def test_every_routine_has_golden_cases():
    from lsmlib_b200 import abi
    syms = {c[1] for c in CASES}
    assert syms == set(abi.SIGNATURES)


# ---- the reference's boundary-condition examples as a property --------------------

import oracle  # noqa: E402
from neumann_property import LIMIT, boundary_errors  # noqa: E402


@pytest.mark.parametrize("scheme", sorted(LIMIT))
@pytest.mark.parametrize("impl", ["reference", "oracle"])
def test_neumann_fill_zeroes_normal_derivatives(impl, scheme):
    if impl == "reference":
        if not oracle.reference_available():
            pytest.skip("oracle/_ref/libref.so not built")
        tb = oracle.reference_toolbox()
    else:
        tb = oracle.oracle_toolbox()
    assert max(boundary_errors(tb.call, scheme)) <= LIMIT[scheme]


def test_heaviside_matches_reference_macro():
    """LSM_HEAVISIDE (lsm_calculus_toolbox.h:41-45), compiled from the
    reference header (oracle/_ref/libcalculus.so), against the oracle's
    restatement that the adjoint loss uses: bit for bit, across the smoothed
    band and past both ends, for two band widths."""
    import ctypes
    import os

    import numpy as np
    path = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libcalculus.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/libcalculus.so not built (make -C oracle ref)")
    lib = ctypes.CDLL(path)
    lib.ref_heaviside.restype = ctypes.c_double
    lib.ref_heaviside.argtypes = [ctypes.c_double, ctypes.c_double]
    for eps in (1.5 / 128, 0.3):
        x = np.concatenate([np.linspace(-2 * eps, 2 * eps, 4001), [-eps, eps, 0.0]])
        ref = np.array([lib.ref_heaviside(v, eps) for v in x])
        assert np.array_equal(ref.view(np.uint64), oracle.heaviside(x, eps).view(np.uint64))
