"""ctypes bindings for the CPU oracles.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` to check (never to produce) results.

Two oracles:

* ``CxOracle`` -- ``libcx_oracle.so``, the C restatement in ``cx_oracle.c``
  (always built by ``make -C oracle oracle``).
* ``RefOracle`` -- ``_ref/libref_prolong.so``, the reference operators
  (CarpetX/src/prolongate_3d_rf2*.cxx) compiled unmodified; present when the
  reference tree was available at build time.
* ``RefBoundary`` -- ``_ref/libref_bc.so``, the reference outer boundary
  conditions (CarpetX/src/boundaries*.cxx) compiled unmodified, same proviso.

Boundary conditions take a ``spec`` dict: ``symmetry`` and ``boundary``
(2 x 3 nested lists of CarpetX's symmetry_t / boundary_t values, [face][dir]),
``domain_lo``/``domain_hi`` (cell-centred domain box), ``prob_lo``,
``prob_hi``, ``dx``, ``indextype`` (1 = cell centred), and per component
``dirichlet``, ``robin`` and ``parity`` (ncomp x 3 of +-1).

Arrays are numpy float64, Fortran-ordered FAB layout flattened as
``(ncomp, nz, ny, nx)`` C-contiguous (x fastest, component stride = box points).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

FAMILIES = {
    # type name -> orders, as registered in CarpetX/src/prolongate_3d_rf2_impl_*.cxx
    "interpolate": (1, 3, 5, 7),
    "conservative": (0, 1),
    "ddf": (1, 3, 5, 7),
    "eno": (3, 5),
    "minmod": (1, 3, 5),
    "hermite": (1, 3, 5),
    "natural": (1, 3, 5, 7),
    "poly-cons3lfb": (1, 3, 5),
    "poly-eno3lfb": (1, 3, 5),
}

_I3 = ctypes.c_int * 3
_DP = ctypes.POINTER(ctypes.c_double)


def _i3(v):
    return _I3(*[int(x) for x in v])


def _dp(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def box_shape(lo, hi):
    """(nz, ny, nx) of the inclusive box [lo, hi]."""
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


_BC_ARGTYPES = [ctypes.c_int * 6, ctypes.c_int * 6, _I3, _I3, ctypes.c_double * 3,
                ctypes.c_double * 3, ctypes.c_double * 3, _I3, ctypes.c_int, _DP, _DP,
                ctypes.POINTER(ctypes.c_int), _DP, _I3, _I3]


def _bc_call(fn, spec, data, lo, hi):
    """Calls a boundary-condition entry with the signature of
    cxo_boundary_box / ref_boundary_box on data (ncomp, nz, ny, nx)."""
    D3 = ctypes.c_double * 3
    ncomp = len(spec["dirichlet"])
    assert data.shape == (ncomp,) + box_shape(lo, hi)
    sym = (ctypes.c_int * 6)(*[int(v) for f in spec["symmetry"] for v in f])
    bc = (ctypes.c_int * 6)(*[int(v) for f in spec["boundary"] for v in f])
    dirv = np.ascontiguousarray(spec["dirichlet"], dtype=np.float64)
    rob = np.ascontiguousarray(spec["robin"], dtype=np.float64)
    par = np.ascontiguousarray(spec["parity"], dtype=np.int32).reshape(-1)
    return fn(sym, bc, _i3(spec["domain_lo"]), _i3(spec["domain_hi"]), D3(*spec["prob_lo"]),
              D3(*spec["prob_hi"]), D3(*spec["dx"]), _i3(spec["indextype"]), ncomp, _dp(dirv),
              _dp(rob), par.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(data), _i3(lo),
              _i3(hi))


class CxOp(ctypes.Structure):
    _fields_ = [("cent", ctypes.c_int * 3), ("intp", ctypes.c_int * 3),
                ("order", ctypes.c_int * 3), ("fb", ctypes.c_int)]


class CxOracle:
    """The C restatement (cx_oracle.c)."""

    def __init__(self, path=None):
        path = path or os.path.join(HERE, "libcx_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run make -C oracle oracle)")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.cxo_lookup.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(CxOp)]
        L.cxo_prolong.argtypes = [ctypes.POINTER(CxOp), ctypes.c_int, _DP, _I3, _I3, _DP, _I3, _I3,
                                  _I3, _I3, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.cxo_prolong_adjoint.argtypes = [ctypes.POINTER(CxOp), ctypes.c_int, _DP, _I3, _I3, _DP,
                                          _I3, _I3, _I3, _I3, ctypes.c_int, _DP]
        L.cxo_restrict.argtypes = [ctypes.c_int, _DP, _I3, _I3, _DP, _I3, _I3, _I3, _I3, ctypes.c_int]
        L.cxo_restrict_adjoint.argtypes = [ctypes.c_int, _DP, _I3, _I3, _DP, _I3, _I3, _I3, _I3,
                                           ctypes.c_int]
        L.cxo_coarse_box.argtypes = [ctypes.POINTER(CxOp), _I3, _I3, _I3, _I3]
        L.cxo_required_ghosts.argtypes = [ctypes.POINTER(CxOp), _I3]
        L.cxo_coeffs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP]
        L.cxo_boundary_box.argtypes = _BC_ARGTYPES

    def op(self, typ, order, indextype):
        o = CxOp()
        if self.lib.cxo_lookup(typ.encode(), order, indextype, ctypes.byref(o)) != 0:
            raise ValueError(f"unknown operator {typ} order {order} indextype {indextype}")
        return o

    def exists(self, typ, order, indextype):
        o = CxOp()
        return self.lib.cxo_lookup(typ.encode(), order, indextype, ctypes.byref(o)) == 0

    def coarse_box(self, typ, order, indextype, flo, fhi):
        o = self.op(typ, order, indextype)
        clo, chi = _I3(), _I3()
        self.lib.cxo_coarse_box(ctypes.byref(o), _i3(flo), _i3(fhi), clo, chi)
        return tuple(clo), tuple(chi)

    def required_ghosts(self, typ, order, indextype):
        o = self.op(typ, order, indextype)
        g = _I3()
        self.lib.cxo_required_ghosts(ctypes.byref(o), g)
        return tuple(g)

    def coeffs(self, cent, intp, order, row=0):
        out = np.zeros(16)
        n = self.lib.cxo_coeffs(cent, intp, order, row, _dp(out))
        return out[:n]

    def prolong(self, typ, order, indextype, per_group, crse, clo, chi, fine, flo, fhi, rlo, rhi,
                ncomp, want_shifts=False):
        o = self.op(typ, order, indextype)
        nreg = int(np.prod(box_shape(rlo, rhi)))
        nblk = 1 if per_group else ncomp
        shifts = np.zeros(3 * nreg * nblk, np.int8) if want_shifts else None
        fb = np.zeros(nreg * nblk, np.uint8) if want_shifts else None
        rc = self.lib.cxo_prolong(ctypes.byref(o), int(per_group), _dp(crse), _i3(clo), _i3(chi),
                                  _dp(fine), _i3(flo), _i3(fhi), _i3(rlo), _i3(rhi), int(ncomp),
                                  shifts.ctypes.data if want_shifts else None,
                                  fb.ctypes.data if want_shifts else None)
        if rc != 0:
            raise ValueError("cxo_prolong rejected its arguments")
        return (shifts, fb) if want_shifts else None

    def prolong_adjoint(self, typ, order, indextype, per_group, crse, clo, chi, fine_bar, flo, fhi,
                        rlo, rhi, ncomp, crse_bar):
        o = self.op(typ, order, indextype)
        rc = self.lib.cxo_prolong_adjoint(ctypes.byref(o), int(per_group), _dp(crse), _i3(clo),
                                          _i3(chi), _dp(fine_bar), _i3(flo), _i3(fhi), _i3(rlo),
                                          _i3(rhi), int(ncomp), _dp(crse_bar))
        if rc != 0:
            raise ValueError("cxo_prolong_adjoint rejected its arguments")

    def restrict(self, indextype, fine, flo, fhi, crse, clo, chi, rlo, rhi, ncomp):
        rc = self.lib.cxo_restrict(int(indextype), _dp(fine), _i3(flo), _i3(fhi), _dp(crse),
                                   _i3(clo), _i3(chi), _i3(rlo), _i3(rhi), int(ncomp))
        if rc != 0:
            raise ValueError("cxo_restrict rejected its arguments")

    def restrict_adjoint(self, indextype, crse_bar, clo, chi, fine_bar, flo, fhi, rlo, rhi, ncomp):
        rc = self.lib.cxo_restrict_adjoint(int(indextype), _dp(crse_bar), _i3(clo), _i3(chi),
                                           _dp(fine_bar), _i3(flo), _i3(fhi), _i3(rlo), _i3(rhi),
                                           int(ncomp))
        if rc != 0:
            raise ValueError("cxo_restrict_adjoint rejected its arguments")


    def boundary(self, spec, data, lo, hi):
        """Outer boundary conditions of one FAB, in place (cxo_boundary_box)."""
        if _bc_call(self.lib.cxo_boundary_box, spec, data, lo, hi) != 0:
            raise ValueError("cxo_boundary_box rejected its arguments")


class RefBoundary:
    """The reference boundary conditions compiled unmodified (oracle/_ref)."""

    PATH = os.path.join(HERE, "_ref", "libref_bc.so")

    def __init__(self):
        if not os.path.exists(self.PATH):
            raise RuntimeError(f"reference oracle not built: {self.PATH}")
        self.lib = ctypes.CDLL(self.PATH)
        self.lib.ref_boundary_box.argtypes = _BC_ARGTYPES

    @classmethod
    def available(cls):
        return os.path.exists(cls.PATH)

    def boundary(self, spec, data, lo, hi):
        """BoundaryCondition(groupdata, dest).apply() on one FAB, in place."""
        if _bc_call(self.lib.ref_boundary_box, spec, data, lo, hi) != 0:
            raise ValueError("ref_boundary_box rejected its arguments")


class RefOracle:
    """The reference operators compiled unmodified (oracle/_ref)."""

    def __init__(self, fast=False):
        name = "libref_prolong_fast.so" if fast else "libref_prolong.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle not built: {path}")
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_prolong.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP,
                                  _I3, _I3, _DP, _I3, _I3, _I3, _I3, ctypes.c_int]
        L.ref_coarse_box.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _I3, _I3, _I3, _I3]
        L.ref_prolong_exists.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int]

    @staticmethod
    def available(fast=False):
        name = "libref_prolong_fast.so" if fast else "libref_prolong.so"
        return os.path.exists(os.path.join(HERE, "_ref", name))

    def exists(self, typ, order, indextype):
        return self.lib.ref_prolong_exists(typ.encode(), order, indextype) == 0

    def coarse_box(self, typ, order, indextype, flo, fhi):
        clo, chi = _I3(), _I3()
        if self.lib.ref_coarse_box(typ.encode(), order, indextype, _i3(flo), _i3(fhi), clo, chi):
            raise ValueError("unknown operator")
        return tuple(clo), tuple(chi)

    def prolong(self, typ, order, indextype, per_group, crse, clo, chi, fine, flo, fhi, rlo, rhi,
                ncomp):
        rc = self.lib.ref_prolong(typ.encode(), order, indextype, int(per_group), _dp(crse),
                                  _i3(clo), _i3(chi), _dp(fine), _i3(flo), _i3(fhi), _i3(rlo),
                                  _i3(rhi), int(ncomp))
        if rc != 0:
            raise ValueError("unknown operator")


def restrict_selection(groups):
    """Time levels Restrict() restricts per group (CarpetX/src/
    schedule.cxx:2717-2837): none for the regrid error (:2746-2747) or a
    group with do_restrict false (:2749-2750); otherwise all but the oldest,
    all of them when the group has one (:2755-2756).  groups: dicts with
    keys ntimelevels, do_restrict and optionally is_regrid_error."""
    out = []
    for g in groups:
        if g.get("is_regrid_error", False) or not g["do_restrict"]:
            out.append(0)
            continue
        n = int(g["ntimelevels"])
        out.append(n - 1 if n > 1 else n)
    return out
