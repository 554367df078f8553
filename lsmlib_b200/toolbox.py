"""Python mirror of the LSMLIB 3D toolbox interface.

``Toolbox(lib, prefix)`` exposes every routine of :mod:`lsmlib_b200.abi` under
the reference's upper-case macro name (``LSM3D_HJ_WENO5`` ...), taking
:class:`Field` objects instead of (pointer, six bounds) pairs.  The argument
meaning is the reference's; errors of the GPU library are raised as
:class:`LsmgpuError` by the caller in :mod:`lsmlib_b200.gpu`.

A :class:`Field` is a column-major (Fortran order) 3D array with the index of
its first element (``lo``); its ghost box is ``lo .. lo + shape - 1``.  The
data is either a numpy array on the host or a :class:`lsmlib_b200.gpu.DeviceArray`.
"""
import ctypes

import numpy as np

from . import abi


class Field:
    """A 3D array with Fortran-order storage and explicit lower bounds."""

    def __init__(self, data, lo=(0, 0, 0)):
        self.data = data
        self.lo = tuple(int(x) for x in lo)
        if isinstance(data, np.ndarray):
            if data.ndim != 3 or not data.flags.f_contiguous:
                raise ValueError("Field data must be a 3D Fortran-ordered array")
        self.shape = tuple(int(x) for x in data.shape)

    @classmethod
    def zeros(cls, lo, hi, dtype=np.float64):
        shape = tuple(h - l + 1 for l, h in zip(lo, hi))
        return cls(np.zeros(shape, dtype=dtype, order="F"), lo)

    @classmethod
    def full(cls, lo, hi, value, dtype=np.float64):
        shape = tuple(h - l + 1 for l, h in zip(lo, hi))
        return cls(np.full(shape, value, dtype=dtype, order="F"), lo)

    @property
    def hi(self):
        return tuple(l + n - 1 for l, n in zip(self.lo, self.shape))

    @property
    def box(self):
        """(ilo, ihi, jlo, jhi, klo, khi)"""
        lo, hi = self.lo, self.hi
        return (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])

    def ptr(self):
        d = self.data
        if isinstance(d, np.ndarray):
            return d.ctypes.data
        return d.ptr

    def copy(self):
        return Field(self.data.copy(order="F"), self.lo)

    def view(self, lo, hi):
        """numpy view of the sub-box [lo, hi] (inclusive, absolute indices)."""
        sl = tuple(slice(l - o, h - o + 1) for l, h, o in zip(lo, hi, self.lo))
        return self.data[sl]


def macro_name(symbol):
    """lsm3dhjweno5_ -> LSM3D_HJ_WENO5 (the reference's header macro name)."""
    return _MACROS[symbol]


_MACROS = {
    "lsm3dhjeno1_": "LSM3D_HJ_ENO1", "lsm3dhjeno2_": "LSM3D_HJ_ENO2",
    "lsm3dhjeno3_": "LSM3D_HJ_ENO3", "lsm3dhjweno5_": "LSM3D_HJ_WENO5",
    "lsm3dupwindhjeno1_": "LSM3D_UPWIND_HJ_ENO1",
    "lsm3dupwindhjeno2_": "LSM3D_UPWIND_HJ_ENO2",
    "lsm3dupwindhjeno3_": "LSM3D_UPWIND_HJ_ENO3",
    "lsm3dupwindhjweno5_": "LSM3D_UPWIND_HJ_WENO5",
    "lsm3dzerooutlevelseteqnrhs_": "LSM3D_ZERO_OUT_LEVEL_SET_EQN_RHS",
    "lsm3daddadvectiontermtolserhs_": "LSM3D_ADD_ADVECTION_TERM_TO_LSE_RHS",
    "lsm3daddnormalveltermtolserhs_": "LSM3D_ADD_NORMAL_VEL_TERM_TO_LSE_RHS",
    "lsm3daddconstnormalveltermtolserhs_": "LSM3D_ADD_CONST_NORMAL_VEL_TERM_TO_LSE_RHS",
    "lsm3dcomputereinitializationeqnrhs_": "LSM3D_COMPUTE_REINITIALIZATION_EQN_RHS",
    "lsm3dcomputefieldextensioneqnrhs_": "LSM3D_COMPUTE_FIELD_EXTENSION_EQN_RHS",
    "lsm3dcomputesignedunitnormal_": "LSM3D_COMPUTE_SIGNED_UNIT_NORMAL",
    "lsm3drk1step_": "LSM3D_RK1_STEP",
    "lsm3dtvdrk2stage1_": "LSM3D_TVD_RK2_STAGE1",
    "lsm3dtvdrk2stage2_": "LSM3D_TVD_RK2_STAGE2",
    "lsm3dtvdrk3stage1_": "LSM3D_TVD_RK3_STAGE1",
    "lsm3dtvdrk3stage2_": "LSM3D_TVD_RK3_STAGE2",
    "lsm3dtvdrk3stage3_": "LSM3D_TVD_RK3_STAGE3",
    "lsm3dmaxnormdiff_": "LSM3D_MAX_NORM_DIFF",
    "lsm3dcomputestableadvectiondt_": "LSM3D_COMPUTE_STABLE_ADVECTION_DT",
    "lsm3dcomputestablenormalveldt_": "LSM3D_COMPUTE_STABLE_NORMAL_VEL_DT",
    "lsm3dcomputestableconstnormalveldt_": "LSM3D_COMPUTE_STABLE_CONST_NORMAL_VEL_DT",
    "lsm3dlinearextrapolation_": "LSM3D_LINEAR_EXTRAPOLATION",
    "lsm3dcopyextrapolation_": "LSM3D_COPY_EXTRAPOLATION",
    "lsm3dhomogeneousneumanneno1_": "LSM3D_HOMOGENEOUS_NEUMANN_ENO1",
    "lsm3dhomogeneousneumanneno2_": "LSM3D_HOMOGENEOUS_NEUMANN_ENO2",
    "lsm3dhomogeneousneumanneno3_": "LSM3D_HOMOGENEOUS_NEUMANN_ENO3",
    "lsm3dhomogeneousneumannweno5_": "LSM3D_HOMOGENEOUS_NEUMANN_WENO5",
    "lsm3dcentralgradorder2_": "LSM3D_CENTRAL_GRAD_ORDER2",
    "lsm3dcentralgradorder4_": "LSM3D_CENTRAL_GRAD_ORDER4",
    "lsm3dlaplacianorder2_": "LSM3D_LAPLACIAN_ORDER2",
    "lsm3dphiupwindgradf_": "LSM3D_PHI_UPWIND_GRAD_F",
    "lsm3daveragegradphi_": "LSM3D_AVERAGE_GRAD_PHI",
    "lsm3dgradientmagnitude_": "LSM3D_GRADIENT_MAGNITUDE",
    "lsm3daddconstcurvtermtolserhs_": "LSM3D_ADD_CONST_CURV_TERM_TO_LSE_RHS",
    "lsm3daddconstprecomputedcurvtermtolserhs_":
        "LSM3D_ADD_CONST_PRECOMPUTED_CURV_TERM_TO_LSE_RHS",
    "lsm3daddexternalandnormalveltermtolserhs_":
        "LSM3D_ADD_EXTERNAL_AND_NORMAL_VEL_TERM_TO_LSE_RHS",
    "lsm3dcomputeorthogonalizationeqnrhs_": "LSM3D_COMPUTE_ORTHOGONALIZATION_EQN_RHS",
    "lsm3dcomputedistanceforsubcellfix_": "LSM3D_COMPUTE_DISTANCE_FOR_SUBCELL_FIX",
    "lsm3dcomputereinitializationeqnrhssubcellfixorder1_":
        "LSM3D_COMPUTE_REINITIALIZATION_EQN_RHS_SUBCELL_FIX_ORDER1",
}


class Toolbox:
    """Callable table of toolbox routines from one shared library.

    ``real`` is the C type of LSMLIB_REAL for that library (double for the
    FP64 build); ``check`` is called after every routine (the GPU library uses
    it to raise on a recorded error)."""

    def __init__(self, lib, prefix="", real=ctypes.c_double, check=None):
        self.lib, self.prefix, self.real, self.check = lib, prefix, real, check
        self._fns = {}
        for sym in abi.SIGNATURES:
            fn = getattr(lib, prefix + sym)
            fn.restype = None
            fn.argtypes = [ctypes.c_void_p] * abi.n_c_args(abi.SIGNATURES[sym])
            self._fns[sym] = fn
        for sym in abi.SIGNATURES:
            setattr(self, _MACROS[sym], self._bind(sym))

    def _bind(self, sym):
        def call(*args, **kw):
            return self.call(sym, *args, **kw)
        call.__name__ = _MACROS[sym]
        return call

    def call(self, sym, fields, fillbox=None, **scalars):
        """Call routine ``sym``.

        ``fields`` maps argument names to :class:`Field`; scratch arrays may be
        omitted (a scratch array with the ``phi`` box is supplied).  ``fillbox``
        is (ilo, ihi, jlo, jhi, klo, khi).  Real scalars and int scalars are
        passed by keyword; outputs ("W:" kinds) are returned in a dict."""
        items = abi.parse(abi.SIGNATURES[sym])
        keep = []          # objects that must outlive the call
        cargs = []
        group = []
        outs = {}
        scratch_like = fields.get("phi") or fields.get("S") or next(iter(fields.values()))
        for kind, name in items:
            if kind in ("I", "O", "X", "S"):
                f = fields.get(name)
                if f is None:
                    if kind != "S":
                        raise TypeError("%s: missing array %s" % (sym, name))
                    f = Field(np.zeros(scratch_like.shape, order="F",
                                       dtype=np.dtype(self.real)),
                              scratch_like.lo)
                    keep.append(f)
                group.append(f)
                cargs.append(f.ptr())
            elif kind == "G":
                box = group[0].box
                for g in group[1:]:
                    if g.box != box:
                        raise ValueError("%s: arrays sharing a ghost box differ" % sym)
                group = []
                for v in box:
                    c = ctypes.c_int(v); keep.append(c)
                    cargs.append(ctypes.addressof(c))
            elif kind == "F":
                if fillbox is None:
                    raise TypeError("%s: fillbox required" % sym)
                for v in fillbox:
                    c = ctypes.c_int(int(v)); keep.append(c)
                    cargs.append(ctypes.addressof(c))
            elif kind == "R":
                c = self.real(scalars[name]); keep.append(c)
                cargs.append(ctypes.addressof(c))
            elif kind == "N":
                c = ctypes.c_int(int(scalars[name])); keep.append(c)
                cargs.append(ctypes.addressof(c))
            elif kind == "W":
                c = self.real(0.0); keep.append(c)
                outs[name] = c
                cargs.append(ctypes.addressof(c))
            else:
                raise ValueError(kind)
        self._fns[sym](*cargs)
        if self.check is not None:
            self.check(sym)
        return {k: v.value for k, v in outs.items()}
