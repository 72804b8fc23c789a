"""carpetx_b200: B200 (sm_100a) refinement-factor-2 transfer operators of CarpetX.

Python bindings over the C ABI of ``include/carpetx_b200.h`` (ctypes), used by
the tests, the benchmark and the autograd wrappers.  FABs are CUDA float64
tensors of shape ``(ncomp, nz, ny, nx)`` (x fastest, component stride = box
points: the amrex::FArrayBox layout); boxes are inclusive ``(lo, hi)`` integer
triples in AMReX index space.

The compiled library ``libcarpetx_b200.so`` must exist next to this file (build
it with ``python -m carpetx_b200.build``); there is no CPU fallback: every
call raises if the library or a CUDA device is missing.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcarpetx_b200.so")

# status codes (include/carpetx_b200.h)
CX_OK, CX_EINVAL, CX_EUNSUPPORTED, CX_ECUDA, CX_ETIMEOUT, CX_ENOMEM, CX_ENODEVICE = range(7)

FAMILIES = {
    # prolongation_type -> orders (CarpetX/src/prolongate_3d_rf2_impl_*.cxx)
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


class CxError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


_I3 = ctypes.c_int * 3
_VP = ctypes.c_void_p
_I = ctypes.c_int
_lib = None


class CxBox(ctypes.Structure):
    """cx_box_t"""
    _fields_ = [("op", ctypes.c_int32), ("ncomp", _I), ("crse", _VP), ("crse_lo", _I3),
                ("crse_hi", _I3), ("fine", _VP), ("fine_lo", _I3), ("fine_hi", _I3),
                ("reg_lo", _I3), ("reg_hi", _I3)]


# symmetries and boundary conditions (CarpetX driver.hxx:41-57)
SYM_NONE, SYM_INTERPATCH, SYM_PERIODIC, SYM_REFLECTION = range(4)
BC_NONE, BC_SYMMETRY_BOUNDARY, BC_DIRICHLET, BC_LINEAR_EXTRAPOLATION, BC_NEUMANN, BC_ROBIN = range(6)
BC_MAX_COMPS = 16
_D3 = ctypes.c_double * 3


class CxBc(ctypes.Structure):
    """cx_bc_t"""
    _fields_ = [("symmetry", _I3 * 2), ("boundary", _I3 * 2), ("domain_lo", _I3),
                ("domain_hi", _I3), ("prob_lo", _D3), ("prob_hi", _D3), ("dx", _D3),
                ("indextype", _I3), ("nghost", _I3), ("ncomp", _I),
                ("dirichlet", ctypes.c_double * BC_MAX_COMPS),
                ("robin", ctypes.c_double * BC_MAX_COMPS), ("parity", _I3 * BC_MAX_COMPS)]


class CxBcFab(ctypes.Structure):
    """cx_bc_fab_t"""
    _fields_ = [("data", _VP), ("lo", _I3), ("hi", _I3)]


class CxRestrictBox(ctypes.Structure):
    """cx_restrict_box_t"""
    _fields_ = [("indextype", _I), ("ncomp", _I), ("fine", _VP), ("fine_lo", _I3),
                ("fine_hi", _I3), ("crse", _VP), ("crse_lo", _I3), ("crse_hi", _I3),
                ("reg_lo", _I3), ("reg_hi", _I3)]


class CxRestrictGroup(ctypes.Structure):
    """cx_restrict_group_t"""
    _fields_ = [("indextype", _I), ("ncomp", _I), ("ntimelevels", _I), ("do_restrict", _I),
                ("is_regrid_error", _I), ("nfabs", _I), ("fabs", ctypes.POINTER(CxRestrictBox))]


class CxFab(ctypes.Structure):
    """cx_fab_t"""
    _fields_ = [("data", _VP), ("lo", _I3), ("hi", _I3), ("valid_lo", _I3), ("valid_hi", _I3)]


def bc_struct(spec):
    """cx_bc_t from a dict: symmetry, boundary ([face][dir] nested lists),
    domain_lo, domain_hi, prob_lo, prob_hi, dx, indextype, nghost (optional,
    default 0) and per component dirichlet, robin, parity (ncomp x 3)."""
    b = CxBc()
    n = len(spec["dirichlet"])
    if not 1 <= n <= BC_MAX_COMPS or len(spec["robin"]) != n or len(spec["parity"]) != n:
        raise ValueError(f"1..{BC_MAX_COMPS} components with dirichlet, robin and parity each")
    for f in range(2):
        b.symmetry[f] = _i3(spec["symmetry"][f])
        b.boundary[f] = _i3(spec["boundary"][f])
    b.domain_lo, b.domain_hi = _i3(spec["domain_lo"]), _i3(spec["domain_hi"])
    b.prob_lo, b.prob_hi = _D3(*spec["prob_lo"]), _D3(*spec["prob_hi"])
    b.dx = _D3(*spec["dx"])
    b.indextype = _i3(spec["indextype"])
    b.nghost = _i3(spec.get("nghost", (0, 0, 0)))
    b.ncomp = n
    for c in range(n):
        b.dirichlet[c] = float(spec["dirichlet"][c])
        b.robin[c] = float(spec["robin"][c])
        b.parity[c] = _i3(spec["parity"][c])
    return b


def lib():
    """The loaded C library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run python -m carpetx_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        L.cx_status_string.restype = ctypes.c_char_p
        L.cx_status_string.argtypes = [_I]
        L.cx_last_error.restype = ctypes.c_char_p
        L.cx_prolong_lookup.argtypes = [ctypes.c_char_p, _I, _I, ctypes.POINTER(ctypes.c_int32)]
        L.cx_prolong_required_ghosts.argtypes = [ctypes.c_int32, _I3]
        L.cx_prolong_coarse_box.argtypes = [ctypes.c_int32, _I3, _I3, _I3, _I3]
        L.cx_prolong_box.argtypes = [ctypes.c_int32, _VP, _I3, _I3, _VP, _I3, _I3, _I3, _I3, _I, _I,
                                     _VP]
        L.cx_prolong_box_diag.argtypes = [ctypes.c_int32, _VP, _I3, _I3, _VP, _I3, _I3, _I3, _I3,
                                          _I, _I, _VP, _VP, _VP]
        L.cx_level_plan_create.argtypes = [ctypes.POINTER(CxBox), _I, _I, ctypes.POINTER(_VP)]
        L.cx_level_plan_create_adjoint.argtypes = [ctypes.POINTER(CxBox), _I, _I,
                                                   ctypes.POINTER(_VP)]
        L.cx_level_plan_create_adjoint_at.argtypes = [ctypes.POINTER(CxBox), ctypes.POINTER(_VP),
                                                      _I, _I, ctypes.POINTER(_VP)]
        L.cx_level_plan_execute.argtypes = [_VP, _VP]
        L.cx_level_plan_stats.argtypes = [_VP, ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(ctypes.c_int64)]
        L.cx_level_plan_launches.argtypes = [_VP, ctypes.POINTER(_I)]
        L.cx_level_plan_destroy.argtypes = [_VP]
        L.cx_restrict_box.argtypes = [_I, _VP, _I3, _I3, _VP, _I3, _I3, _I3, _I3, _I, _VP]
        L.cx_restrict_adjoint_box.argtypes = [_I, _VP, _I3, _I3, _VP, _I3, _I3, _I3, _I3, _I, _VP]
        L.cx_prolong_adjoint_box.argtypes = [ctypes.c_int32, _VP, _I3, _I3, _VP, _I3, _I3, _I3,
                                             _I3, _I, _I, _VP, _VP]
        L.cx_boundary_box.argtypes = [ctypes.POINTER(CxBc), _VP, _I3, _I3, _VP]
        L.cx_boundary_plan_create.argtypes = [ctypes.POINTER(CxBc), ctypes.POINTER(CxBcFab), _I,
                                              ctypes.POINTER(_VP)]
        L.cx_boundary_plan_execute.argtypes = [_VP, _VP]
        L.cx_boundary_plan_stats.argtypes = [_VP, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(ctypes.c_int64)]
        L.cx_boundary_plan_destroy.argtypes = [_VP]
        L.cx_copy_plan_parallel_copy.argtypes = [ctypes.POINTER(CxFab), _I, ctypes.POINTER(CxFab),
                                                 _I, _I, _I3, _I3, _I3, ctypes.POINTER(_VP)]
        L.cx_copy_plan_fill_boundary.argtypes = [ctypes.POINTER(CxFab), _I, _I, _I3, _I3,
                                                 ctypes.POINTER(_VP)]
        L.cx_copy_plan_execute.argtypes = [_VP, _VP]
        L.cx_copy_plan_stats.argtypes = [_VP, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64)]
        L.cx_copy_plan_destroy.argtypes = [_VP]
        L.cx_reflux_plan_create.argtypes = [ctypes.POINTER(CxFab), _I,
                                            ctypes.POINTER(ctypes.POINTER(CxFab)),
                                            ctypes.POINTER(ctypes.POINTER(CxFab)), _I, _I,
                                            ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                            ctypes.POINTER(_VP)]
        L.cx_reflux_plan_execute.argtypes = [_VP, _VP]
        L.cx_reflux_plan_stats.argtypes = [_VP, ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(_I)]
        L.cx_reflux_plan_destroy.argtypes = [_VP]
        L.cx_restrict_plan_create.argtypes = [ctypes.POINTER(CxRestrictBox), _I,
                                              ctypes.POINTER(_VP)]
        L.cx_restrict_plan_execute.argtypes = [_VP, _VP]
        L.cx_restrict_plan_stats.argtypes = [_VP, ctypes.POINTER(ctypes.c_int64),
                                             ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(_I)]
        L.cx_restrict_plan_destroy.argtypes = [_VP]
        L.cx_restrict_groups_plan_create.argtypes = [ctypes.POINTER(CxRestrictGroup), _I,
                                                     ctypes.POINTER(_I), ctypes.POINTER(_VP)]
        L.cx_debug_set_wait_limit.argtypes = [ctypes.c_longlong]
        L.cx_debug_stream_kind.argtypes = [ctypes.c_int32]
        L.cx_debug_set_stream_schedule.argtypes = [_I, _I, _I]
        _lib = L
    return _lib


def _check(status):
    if status != CX_OK:
        L = lib()
        raise CxError(status, f"{L.cx_status_string(status).decode()}: "
                              f"{L.cx_last_error().decode()}")


def _i3(v):
    return _I3(*[int(x) for x in v])


def box_shape(lo, hi):
    """(nz, ny, nx) of the inclusive box [lo, hi]."""
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t, ncomp, lo, hi, what):
    import torch
    if not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or not t.is_cuda:
        raise TypeError(f"{what} must be a CUDA float64 tensor")
    if not t.is_contiguous() or t.numel() < ncomp * _npts(lo, hi):
        raise ValueError(f"{what} must be contiguous with ncomp x box points elements")
    return ctypes.c_void_p(t.data_ptr())


def _npts(lo, hi):
    n = 1
    for a, b in zip(lo, hi):
        n *= max(0, int(b) - int(a) + 1)
    return n


class Op:
    """A prolongation operator: (prolongation_type, order, indextype)."""

    def __init__(self, typ, order, indextype):
        h = ctypes.c_int32()
        _check(lib().cx_prolong_lookup(typ.encode(), int(order), int(indextype), ctypes.byref(h)))
        self.handle = h.value
        self.type, self.order, self.indextype = typ, int(order), int(indextype)

    def required_ghosts(self):
        g = _I3()
        _check(lib().cx_prolong_required_ghosts(self.handle, g))
        return tuple(g)

    def coarse_box(self, fine_lo, fine_hi):
        lo, hi = _I3(), _I3()
        _check(lib().cx_prolong_coarse_box(self.handle, _i3(fine_lo), _i3(fine_hi), lo, hi))
        return tuple(lo), tuple(hi)

    def __repr__(self):
        return f"Op({self.type!r}, {self.order}, {self.indextype})"


def prolong_box(op, crse, crse_lo, crse_hi, fine, fine_lo, fine_hi, reg_lo, reg_hi, ncomp,
                per_group=False, stream=None, shifts=None, fallback=None):
    """cx_prolong_box / cx_prolong_box_diag on CUDA tensors (asynchronous)."""
    L = lib()
    args = (op.handle, _ptr(crse, ncomp, crse_lo, crse_hi, "crse"), _i3(crse_lo), _i3(crse_hi),
            _ptr(fine, ncomp, fine_lo, fine_hi, "fine"), _i3(fine_lo), _i3(fine_hi), _i3(reg_lo),
            _i3(reg_hi), int(ncomp), int(bool(per_group)))
    if shifts is None and fallback is None:
        _check(L.cx_prolong_box(*args, _stream(stream)))
    else:
        _check(L.cx_prolong_box_diag(
            *args, ctypes.c_void_p(shifts.data_ptr() if shifts is not None else 0),
            ctypes.c_void_p(fallback.data_ptr() if fallback is not None else 0), _stream(stream)))


def restrict_box(indextype, fine, fine_lo, fine_hi, crse, crse_lo, crse_hi, reg_lo, reg_hi, ncomp,
                 stream=None):
    """cx_restrict_box on CUDA tensors (asynchronous)."""
    _check(lib().cx_restrict_box(int(indextype), _ptr(fine, ncomp, fine_lo, fine_hi, "fine"),
                                 _i3(fine_lo), _i3(fine_hi),
                                 _ptr(crse, ncomp, crse_lo, crse_hi, "crse"), _i3(crse_lo),
                                 _i3(crse_hi), _i3(reg_lo), _i3(reg_hi), int(ncomp),
                                 _stream(stream)))


def prolong_adjoint_box(op, crse, crse_lo, crse_hi, fine_bar, fine_lo, fine_hi, reg_lo, reg_hi,
                        ncomp, crse_bar, per_group=False, stream=None):
    """cx_prolong_adjoint_box: crse_bar = P^T fine_bar (asynchronous)."""
    _check(lib().cx_prolong_adjoint_box(
        op.handle, _ptr(crse, ncomp, crse_lo, crse_hi, "crse"), _i3(crse_lo), _i3(crse_hi),
        _ptr(fine_bar, ncomp, fine_lo, fine_hi, "fine_bar"), _i3(fine_lo), _i3(fine_hi),
        _i3(reg_lo), _i3(reg_hi), int(ncomp), int(bool(per_group)),
        _ptr(crse_bar, ncomp, crse_lo, crse_hi, "crse_bar"), _stream(stream)))


def restrict_adjoint_box(indextype, crse_bar, crse_lo, crse_hi, fine_bar, fine_lo, fine_hi,
                         reg_lo, reg_hi, ncomp, stream=None):
    """cx_restrict_adjoint_box: fine_bar = R^T crse_bar (asynchronous)."""
    _check(lib().cx_restrict_adjoint_box(
        int(indextype), _ptr(crse_bar, ncomp, crse_lo, crse_hi, "crse_bar"), _i3(crse_lo),
        _i3(crse_hi), _ptr(fine_bar, ncomp, fine_lo, fine_hi, "fine_bar"), _i3(fine_lo),
        _i3(fine_hi), _i3(reg_lo), _i3(reg_hi), int(ncomp), _stream(stream)))


def boundary_box(spec, data, lo, hi, stream=None):
    """cx_boundary_box: the outer boundary conditions of one FAB, in place
    (asynchronous).  spec as for bc_struct."""
    b = bc_struct(spec)
    _check(lib().cx_boundary_box(ctypes.byref(b), _ptr(data, b.ncomp, lo, hi, "data"), _i3(lo),
                                 _i3(hi), _stream(stream)))


class BoundaryPlan:
    """cx_boundary_plan_*: the outer boundary conditions of every FAB of a
    level (GroupData::apply_boundary_conditions) as one launch.  fabs:
    iterable of (tensor, lo, hi); the plan keeps the tensors alive."""

    def __init__(self, spec, fabs):
        b = bc_struct(spec)
        fabs = list(fabs)
        arr = (CxBcFab * max(1, len(fabs)))()
        self._keep = []
        for i, (t, lo, hi) in enumerate(fabs):
            arr[i] = CxBcFab(_ptr(t, b.ncomp, lo, hi, "fab").value, _i3(lo), _i3(hi))
            self._keep.append(t)
        h = ctypes.c_void_p()
        _check(lib().cx_boundary_plan_create(ctypes.byref(b), arr, len(fabs), ctypes.byref(h)))
        self.handle = h

    def execute(self, stream=None):
        _check(lib().cx_boundary_plan_execute(self.handle, _stream(stream)))

    def stats(self):
        a, c = ctypes.c_int64(), ctypes.c_int64()
        _check(lib().cx_boundary_plan_stats(self.handle, ctypes.byref(a), ctypes.byref(c)))
        return {"points": a.value, "bytes": c.value}

    def close(self):
        if self.handle:
            lib().cx_boundary_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _restrict_boxes(boxes, keep):
    arr = (CxRestrictBox * max(1, len(boxes)))()
    for i, b in enumerate(boxes):
        n = int(b["ncomp"])
        arr[i] = CxRestrictBox(int(b["indextype"]), n,
                               _ptr(b["fine"], n, b["fine_lo"], b["fine_hi"], "fine").value,
                               _i3(b["fine_lo"]), _i3(b["fine_hi"]),
                               _ptr(b["crse"], n, b["crse_lo"], b["crse_hi"], "crse").value,
                               _i3(b["crse_lo"]), _i3(b["crse_hi"]), _i3(b["reg_lo"]),
                               _i3(b["reg_hi"]))
        keep += [b["fine"], b["crse"]]
    return arr


class RestrictPlan:
    """cx_restrict_plan_*: the restriction of a whole level (every FAB pair,
    all components) in one launch per index type.  boxes: dicts with keys
    indextype, ncomp, fine, fine_lo, fine_hi, crse, crse_lo, crse_hi, reg_lo,
    reg_hi (tensors as for restrict_box); the plan keeps the tensors alive."""

    def __init__(self, boxes):
        boxes = list(boxes)
        self._keep = []
        arr = _restrict_boxes(boxes, self._keep)
        h = ctypes.c_void_p()
        _check(lib().cx_restrict_plan_create(arr, len(boxes), ctypes.byref(h)))
        self.handle = h
        self.restricted = None

    @classmethod
    def for_groups(cls, groups):
        """cx_restrict_groups_plan_create: Restrict() of one level
        (CarpetX/src/schedule.cxx:2717-2837).  groups: dicts with keys
        indextype, ncomp, ntimelevels, do_restrict, is_regrid_error and fabs
        (per time level, newest first, a list of FAB-pair dicts as for the
        constructor; every time level has the same number of pairs).  The
        plan's `restricted` lists, per group, how many time levels it
        restricts (0 for a skipped group)."""
        groups = list(groups)
        self = cls.__new__(cls)
        self._keep = []
        garr = (CxRestrictGroup * max(1, len(groups)))()
        self._arrays = []
        for g, gr in enumerate(groups):
            tls = list(gr["fabs"])
            nf = len(tls[0]) if tls else 0
            if any(len(t) != nf for t in tls):
                raise ValueError(f"group {g}: every time level needs the same FAB pairs")
            flat = [b for t in tls for b in t]
            arr = _restrict_boxes(flat, self._keep)
            self._arrays.append(arr)
            garr[g] = CxRestrictGroup(int(gr["indextype"]), int(gr["ncomp"]),
                                      int(gr["ntimelevels"]), int(bool(gr["do_restrict"])),
                                      int(bool(gr.get("is_regrid_error", False))), nf,
                                      ctypes.cast(arr, ctypes.POINTER(CxRestrictBox)))
        nres = (_I * max(1, len(groups)))()
        h = ctypes.c_void_p()
        _check(lib().cx_restrict_groups_plan_create(garr, len(groups), nres, ctypes.byref(h)))
        self.handle = h
        self.restricted = [int(nres[g]) for g in range(len(groups))]
        return self

    def execute(self, stream=None):
        _check(lib().cx_restrict_plan_execute(self.handle, _stream(stream)))

    def stats(self):
        a, b, n = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
        _check(lib().cx_restrict_plan_stats(self.handle, ctypes.byref(a), ctypes.byref(b),
                                            ctypes.byref(n)))
        return {"coarse_values": a.value, "bytes": b.value, "launches": n.value}

    def close(self):
        if self.handle:
            lib().cx_restrict_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CopyPlan:
    """cx_copy_plan_*: AMReX's FillBoundary or ParallelCopy of a level as one
    launch.  FABs are tuples (tensor, lo, hi, valid_lo, valid_hi); the plan
    keeps the tensors alive.  Build with CopyPlan.fill_boundary or
    CopyPlan.parallel_copy."""

    def __init__(self, handle, keep):
        self.handle, self._keep = handle, keep

    @staticmethod
    def _fabs(fabs, ncomp):
        arr = (CxFab * max(1, len(fabs)))()
        for i, (t, lo, hi, vlo, vhi) in enumerate(fabs):
            arr[i] = CxFab(_ptr(t, ncomp, lo, hi, "fab").value, _i3(lo), _i3(hi), _i3(vlo),
                           _i3(vhi))
        return arr

    @classmethod
    def fill_boundary(cls, fabs, ncomp, nghost, period=(0, 0, 0)):
        fabs = list(fabs)
        h = ctypes.c_void_p()
        _check(lib().cx_copy_plan_fill_boundary(cls._fabs(fabs, ncomp), len(fabs), int(ncomp),
                                                _i3(nghost), _i3(period), ctypes.byref(h)))
        return cls(h, [f[0] for f in fabs])

    @classmethod
    def parallel_copy(cls, dst, src, ncomp, src_nghost=(0, 0, 0), dst_nghost=(0, 0, 0),
                      period=(0, 0, 0)):
        dst, src = list(dst), list(src)
        h = ctypes.c_void_p()
        _check(lib().cx_copy_plan_parallel_copy(cls._fabs(dst, ncomp), len(dst),
                                                cls._fabs(src, ncomp), len(src), int(ncomp),
                                                _i3(src_nghost), _i3(dst_nghost), _i3(period),
                                                ctypes.byref(h)))
        return cls(h, [f[0] for f in dst + src])

    def execute(self, stream=None):
        _check(lib().cx_copy_plan_execute(self.handle, _stream(stream)))

    def stats(self):
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().cx_copy_plan_stats(self.handle, ctypes.byref(a), ctypes.byref(b),
                                        ctypes.byref(c)))
        return {"points": a.value, "pieces": b.value, "bytes": c.value}

    def close(self):
        if self.handle:
            lib().cx_copy_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LevelPlan:
    """cx_level_plan_*: a whole level transfer as one persistent launch.

    boxes: iterable of dicts with keys op, ncomp, crse, crse_lo, crse_hi, fine,
    fine_lo, fine_hi, reg_lo, reg_hi (tensors as for prolong_box).  The plan
    keeps references to the tensors so their memory outlives it.  With
    adjoint=True (cx_level_plan_create_adjoint) executing the plan overwrites
    every crse tensor with P^T of its fine tensor (region points only); a
    box of a limited operator (ENO, minmod, linear fallback) also carries
    crse_at, the coarse data it is linearised at
    (cx_level_plan_create_adjoint_at)."""

    def __init__(self, boxes, per_group=False, adjoint=False):
        self._keep = []
        arr = (CxBox * max(1, len(boxes)))()
        for i, b in enumerate(boxes):
            n = int(b["ncomp"])
            arr[i] = CxBox(b["op"].handle, n,
                           _ptr(b["crse"], n, b["crse_lo"], b["crse_hi"], "crse").value,
                           _i3(b["crse_lo"]), _i3(b["crse_hi"]),
                           _ptr(b["fine"], n, b["fine_lo"], b["fine_hi"], "fine").value,
                           _i3(b["fine_lo"]), _i3(b["fine_hi"]), _i3(b["reg_lo"]),
                           _i3(b["reg_hi"]))
            self._keep += [b["crse"], b["fine"]]
        h = ctypes.c_void_p()
        if adjoint and any(b.get("crse_at") is not None for b in boxes):
            # the limited operators' linearisation points (cx_level_plan_create_adjoint_at)
            at = (_VP * max(1, len(boxes)))()
            for i, b in enumerate(boxes):
                if b.get("crse_at") is not None:
                    n = int(b["ncomp"])
                    at[i] = _ptr(b["crse_at"], n, b["crse_lo"], b["crse_hi"], "crse_at").value
                    self._keep.append(b["crse_at"])
            _check(lib().cx_level_plan_create_adjoint_at(arr, at, len(boxes), int(bool(per_group)),
                                                         ctypes.byref(h)))
        else:
            create = lib().cx_level_plan_create_adjoint if adjoint else lib().cx_level_plan_create
            _check(create(arr, len(boxes), int(bool(per_group)), ctypes.byref(h)))
        self.handle = h

    def execute(self, stream=None):
        _check(lib().cx_level_plan_execute(self.handle, _stream(stream)))

    def stats(self):
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().cx_level_plan_stats(self.handle, ctypes.byref(a), ctypes.byref(b),
                                         ctypes.byref(c)))
        n = ctypes.c_int()
        _check(lib().cx_level_plan_launches(self.handle, ctypes.byref(n)))
        return {"tiles": a.value, "fine_points": b.value, "bytes": c.value, "launches": n.value}

    def close(self):
        if self.handle:
            lib().cx_level_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefluxPlan:
    """cx_reflux_plan_*: the reflux of a coarse level from the next finer
    one (CarpetX's Reflux(), AMReX FluxRegister semantics).  crse: the
    coarse state FABs; crse_flux[d]: per direction the coarse flux FABs (one
    per state FAB); fine_flux[d]: per direction the fine flux FABs (one per
    fine box); each FAB a tuple (tensor, lo, hi, valid_lo, valid_hi) as for
    CopyPlan.  dx: the coarse cell size; the plan keeps the tensors alive."""

    def __init__(self, crse, crse_flux, fine_flux, ncomp, dx, scale=1.0):
        self._keep = []
        arr_c = CopyPlan._fabs(list(crse), ncomp)
        self._keep.append(arr_c)
        cf = (ctypes.POINTER(CxFab) * 3)()
        ff = (ctypes.POINTER(CxFab) * 3)()
        nfine = len(fine_flux[0])
        for d in range(3):
            a = CopyPlan._fabs(list(crse_flux[d]), ncomp)
            b = CopyPlan._fabs(list(fine_flux[d]), ncomp)
            self._keep += [a, b]
            cf[d] = ctypes.cast(a, ctypes.POINTER(CxFab))
            ff[d] = ctypes.cast(b, ctypes.POINTER(CxFab))
        self._keep += [f[0] for f in crse] + [f[0] for d in range(3) for f in crse_flux[d]]
        self._keep += [f[0] for d in range(3) for f in fine_flux[d]]
        h = ctypes.c_void_p()
        _check(lib().cx_reflux_plan_create(arr_c, len(crse), cf, ff, nfine, int(ncomp),
                                           (ctypes.c_double * 3)(*dx), float(scale),
                                           ctypes.byref(h)))
        self.handle = h

    def execute(self, stream=None):
        _check(lib().cx_reflux_plan_execute(self.handle, _stream(stream)))

    def stats(self):
        a, b, n = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
        _check(lib().cx_reflux_plan_stats(self.handle, ctypes.byref(a), ctypes.byref(b),
                                          ctypes.byref(n)))
        return {"faces": a.value, "bytes": b.value, "launches": n.value}

    def close(self):
        if self.handle:
            lib().cx_reflux_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
