"""CPU checkers for the LSMLIB 3D toolbox hot path (test infrastructure only).

* ``oracle_toolbox()`` -- the hand-written C restatement (lsm_oracle.c), built
  by ``make -C oracle`` into ``oracle/_build/liboracle.so``;
* ``oracle_fmm()`` -- the C restatement of the fast marching method's distance
  function (fmm_oracle.c), in the same library;
* ``reference_toolbox()`` -- the reference's own Fortran routines, translated
  by ``oracle/f77toc.py`` and built by ``make -C oracle ref`` into
  ``oracle/_ref/libref.so`` (needs the reference sources at build time only);
* ``reference_fmm()`` -- the reference's own C fast marching method
  (``computeDistanceFunction3d``), built by ``make -C oracle ref`` into
  ``oracle/_ref/libfmm.so``.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this
package; the product path in lsmlib_b200/ never does.
"""
import ctypes
import os

from lsmlib_b200.toolbox import Toolbox

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")
FMM_SO = os.path.join(HERE, "_ref", "libfmm.so")


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


def fmm_available():
    return os.path.exists(FMM_SO)


def _distance_fn(fn, name):
    import numpy as np
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]

    def run(phi, order, dx, mask=None):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.zeros_like(phi)
        dims = np.array(phi.shape[::-1], dtype=np.intc)
        h = np.array(dx, dtype=np.float64)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        rc = fn(out.ctypes.data, phi.ctypes.data, None if m is None else m.ctypes.data,
                int(order), dims.ctypes.data, h.ctypes.data)
        if rc != 0:
            raise RuntimeError("%s returned %d" % (name, rc))
        return out
    return run


def reference_fmm():
    """The reference's computeDistanceFunction3d (lsm_fast_marching_method.h:
    386-392) as ``f(phi, order, dx, mask=None) -> distance`` on C-ordered
    (nz, ny, nx) numpy arrays (x fastest in memory), dx in x, y, z order."""
    return _distance_fn(_load(FMM_SO).computeDistanceFunction3d, "computeDistanceFunction3d")


def oracle_fmm(ordered=False):
    """The C restatement of the same heap march (fmm_oracle.c), same call.
    ``ordered``: the march popping exact key ties by (acceptance time, index),
    which is what the GPU solver computes; without ties it is the reference's
    march."""
    nm = "orc_computeDistanceFunction3d" + ("_ordered" if ordered else "")
    return _distance_fn(getattr(oracle_lib(), nm), nm)


def _extension_fn(fn, name):
    import numpy as np
    P = ctypes.c_void_p
    fn.restype = ctypes.c_int
    fn.argtypes = [P, P, P, P, P, P, ctypes.c_int, ctypes.c_int, P, P]

    def run(phi, sources, order, dx, mask=None, ext_mask=None):
        """(distance, [extension fields]) for C-ordered (nz, ny, nx) arrays."""
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        srcs = [np.ascontiguousarray(s, dtype=np.float64) for s in sources]
        outs = [np.zeros_like(phi) for _ in srcs]
        dist = np.zeros_like(phi)
        nf = len(srcs)
        src_p = (ctypes.c_void_p * max(nf, 1))(*[s.ctypes.data for s in srcs])
        out_p = (ctypes.c_void_p * max(nf, 1))(*[o.ctypes.data for o in outs])
        dims = np.array(phi.shape[::-1], dtype=np.intc)
        h = np.array(dx, dtype=np.float64)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        em = None if ext_mask is None else np.ascontiguousarray(ext_mask, dtype=np.float64)
        rc = fn(dist.ctypes.data, ctypes.cast(out_p, P), phi.ctypes.data,
                None if m is None else m.ctypes.data, ctypes.cast(src_p, P),
                None if em is None else em.ctypes.data, nf, int(order), dims.ctypes.data,
                h.ctypes.data)
        if rc != 0:
            raise RuntimeError("%s returned %d" % (name, rc))
        return dist, outs
    return run


def reference_extension():
    """The reference's computeExtensionFields3d (lsm_fast_marching_method.h:
    331-341) as ``f(phi, sources, order, dx, mask=None, ext_mask=None) ->
    (distance, [fields])``, C-ordered arrays, dx in x, y, z order."""
    return _extension_fn(_load(FMM_SO).computeExtensionFields3d, "computeExtensionFields3d")


def oracle_extension(ordered=False):
    """The C restatement of the same march with extension fields, same call
    (``ordered`` as for oracle_fmm)."""
    nm = "orc_computeExtensionFields3d" + ("_ordered" if ordered else "")
    return _extension_fn(getattr(oracle_lib(), nm), nm)


def _eikonal_fn(fn, name):
    import numpy as np
    P = ctypes.c_void_p
    fn.restype = ctypes.c_int
    fn.argtypes = [P, P, P, ctypes.c_int, P, P]

    def run(phi, speed, order, dx, mask=None):
        """The solution for boundary data ``phi`` (C-ordered (nz, ny, nx),
        front where phi > -1e-11); a new array."""
        out = np.array(phi, dtype=np.float64, order="C", copy=True)
        f = np.ascontiguousarray(speed, dtype=np.float64)
        dims = np.array(out.shape[::-1], dtype=np.intc)
        h = np.array(dx, dtype=np.float64)
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
        rc = fn(out.ctypes.data, f.ctypes.data, None if m is None else m.ctypes.data,
                int(order), dims.ctypes.data, h.ctypes.data)
        if rc != 0:
            raise RuntimeError("%s returned %d" % (name, rc))
        return out
    return run


def reference_eikonal():
    """The reference's solveEikonalEquation3d (lsm_fast_marching_method.h:
    463-469) as ``f(phi, speed, order, dx, mask=None) -> phi``."""
    return _eikonal_fn(_load(FMM_SO).solveEikonalEquation3d, "solveEikonalEquation3d")


def oracle_eikonal(ordered=False):
    """The C restatement of the same march (fmm_oracle.c), same call
    (``ordered`` as for oracle_fmm)."""
    nm = "orc_solveEikonalEquation3d" + ("_ordered" if ordered else "")
    return _eikonal_fn(getattr(oracle_lib(), nm), nm)


def heaviside(x, eps):
    """LSM_HEAVISIDE of lsm_calculus_toolbox.h:41-45, elementwise (numpy)."""
    import numpy as np
    x = np.asarray(x, dtype=np.float64)
    h = 0.5 * (1 + x / eps + 1 / np.pi * np.sin(np.pi * x / eps))
    return np.where(x < -eps, 0.0, np.where(x > eps, 1.0, h))
