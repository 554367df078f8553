"""The reference's boundary-condition examples as a property of the GPU
routines: after a homogeneous Neumann fill the normal one-sided derivatives
vanish at the boundary (tests/neumann_property.py; the same holds for the
reference's own routines and the oracle in test_oracle_golden.py).  Host
arrays through the C ABI.  Collected after the other GPU parity tests."""
import pytest

from neumann_property import LIMIT, boundary_errors

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme", sorted(LIMIT))
def test_neumann_fill_zeroes_normal_derivatives_on_gpu(scheme):
    from lsmlib_b200 import gpu
    assert max(boundary_errors(gpu.toolbox().call, scheme)) <= LIMIT[scheme]
