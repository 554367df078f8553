"""CPU checkers for the LSMLIB 3D toolbox hot path (test infrastructure only).

* ``oracle_toolbox()`` -- the hand-written C restatement (lsm_oracle.c), built
  by ``make -C oracle`` into ``oracle/_build/liboracle.so``;
* ``reference_toolbox()`` -- the reference's own Fortran routines, translated
  by ``oracle/f77toc.py`` and built by ``make -C oracle ref`` into
  ``oracle/_ref/libref.so`` (needs the reference sources at build time only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this
package; the product path in lsmlib_b200/ never does.
"""
import ctypes
import os

from lsmlib_b200.toolbox import Toolbox

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError("%s not built (run make -C oracle all ref)" % path)
    return ctypes.CDLL(path)


def oracle_lib():
    return _load(ORACLE_SO)


def oracle_toolbox():
    return Toolbox(oracle_lib(), prefix="orc_")


def reference_available():
    return os.path.exists(REF_SO)


def reference_toolbox():
    return Toolbox(_load(REF_SO), prefix="ref_")


def heaviside(x, eps):
    """LSM_HEAVISIDE of lsm_calculus_toolbox.h:41-45, elementwise (numpy)."""
    import numpy as np
    x = np.asarray(x, dtype=np.float64)
    h = 0.5 * (1 + x / eps + 1 / np.pi * np.sin(np.pi * x / eps))
    return np.where(x < -eps, 0.0, np.where(x > eps, 1.0, h))
