"""CPU tests of the C ABI library: it loads, exports every entry point that
include/*.h declares, and its host-side logic (operator registry, CoarseBox,
argument validation, status codes) matches the reference without a GPU."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import carpetx_b200 as cb
from helpers import ALL_OPS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(cx_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = cb.lib()
    names = declared_symbols()
    assert len(names) >= 14
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/ but not exported"


def test_lookup_covers_reference_tables(cx):
    for typ, order, it in ALL_OPS:
        op = cb.Op(typ, order, it)
        assert op.required_ghosts() == cx.required_ghosts(typ, order, it)
        for flo, fhi in [((0, 0, 0), (7, 7, 7)), ((-3, -1, 5), (4, 0, 9)), ((-8, -7, -6), (-1, -2, -3))]:
            assert op.coarse_box(flo, fhi) == cx.coarse_box(typ, order, it, flo, fhi)


def test_lookup_matches_reference_build(ref):
    for typ, order, it in ALL_OPS:
        op = cb.Op(typ, order, it)
        assert op.coarse_box((-5, 0, 3), (10, 9, 4)) == ref.coarse_box(typ, order, it, (-5, 0, 3),
                                                                       (10, 9, 4))


@pytest.mark.parametrize("typ,order,it", [("interpolate", 2, 0), ("conservative", 2, 7),
                                          ("eno", 1, 7), ("nosuch", 1, 0), ("natural", 9, 0),
                                          ("natural", 1, 8), ("natural", 1, -1)])
def test_unknown_operator_is_unsupported(typ, order, it):
    with pytest.raises(cb.CxError) as e:
        cb.Op(typ, order, it)
    assert e.value.status == cb.CX_EUNSUPPORTED


def _raw_prolong(op, clo, chi, flo, fhi, rlo, rhi, ncomp, per_group=0):
    """Call cx_prolong_box with dummy (never dereferenced) device pointers:
    validation happens before any device access."""
    L = cb.lib()
    I3 = ctypes.c_int * 3
    return L.cx_prolong_box(op.handle, ctypes.c_void_p(0x1000), I3(*clo), I3(*chi),
                            ctypes.c_void_p(0x2000), I3(*flo), I3(*fhi), I3(*rlo), I3(*rhi),
                            ncomp, per_group, None)


def test_validation_errors():
    op = cb.Op("interpolate", 3, 0)
    good = dict(clo=(-1, -1, -1), chi=(33, 33, 33), flo=(0, 0, 0), fhi=(63, 63, 63),
                rlo=(0, 0, 0), rhi=(63, 63, 63))
    # region outside the fine box
    bad = dict(good, rhi=(64, 63, 63))
    assert _raw_prolong(op, *bad.values(), 1) == cb.CX_EINVAL
    # coarse box too small: off-1 point 63 reads coarse 30..33
    bad = dict(good, chi=(32, 33, 33))
    assert _raw_prolong(op, *bad.values(), 1) == cb.CX_EINVAL
    assert "does not contain" in cb.lib().cx_last_error().decode()
    bad = dict(good, clo=(0, -1, -1))
    assert _raw_prolong(op, *bad.values(), 1) == cb.CX_EINVAL
    # negative ncomp, too many components per group
    assert _raw_prolong(op, *good.values(), -1) == cb.CX_EINVAL
    assert _raw_prolong(op, *good.values(), 17, per_group=1) == cb.CX_EINVAL
    # empty region or no components: nothing to do, no device needed
    assert _raw_prolong(op, *dict(good, rhi=(-1, 63, 63)).values(), 1) == cb.CX_OK
    assert _raw_prolong(op, *good.values(), 0) == cb.CX_OK


def test_valid_call_without_device_reports_nodevice():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    op = cb.Op("interpolate", 3, 0)
    st = _raw_prolong(op, (-1, -1, -1), (33, 33, 33), (0, 0, 0), (63, 63, 63), (0, 0, 0),
                      (63, 63, 63), 1)
    assert st == cb.CX_ENODEVICE


def test_restrict_validation():
    L = cb.lib()
    I3 = ctypes.c_int * 3
    p = ctypes.c_void_p(0x1000)
    # children of coarse point 4 in a cell direction are 8, 9: fine box must reach 9
    st = L.cx_restrict_box(7, p, I3(0, 0, 0), I3(8, 9, 9), p, I3(0, 0, 0), I3(4, 4, 4),
                           I3(0, 0, 0), I3(4, 4, 4), 1, None)
    assert st == cb.CX_EINVAL
    assert L.cx_restrict_box(8, p, I3(0, 0, 0), I3(9, 9, 9), p, I3(0, 0, 0), I3(4, 4, 4),
                             I3(0, 0, 0), I3(4, 4, 4), 1, None) == cb.CX_EUNSUPPORTED


def test_status_strings():
    L = cb.lib()
    for s in range(7):
        assert L.cx_status_string(s)
