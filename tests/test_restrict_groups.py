"""Restrict() of one level (CarpetX/src/schedule.cxx:2717-2837): the
oracle's group and time-level selection, and the host-side argument checks
of cx_restrict_groups_plan_create (no device work)."""
import ctypes

import carpetx_b200 as cb
from oracle.oracle import restrict_selection


def test_selection_follows_restrict():
    groups = [dict(ntimelevels=1, do_restrict=True), dict(ntimelevels=2, do_restrict=True),
              dict(ntimelevels=3, do_restrict=True), dict(ntimelevels=3, do_restrict=False),
              dict(ntimelevels=1, do_restrict=True, is_regrid_error=True),
              dict(ntimelevels=0, do_restrict=True)]
    assert restrict_selection(groups) == [1, 1, 2, 0, 0, 0]


def _box(indextype, ncomp):
    b = cb.CxRestrictBox()
    b.indextype, b.ncomp = indextype, ncomp
    b.fine, b.crse = 8, 16  # never dereferenced: the checks fail first
    b.fine_lo, b.fine_hi = cb._i3((0, 0, 0)), cb._i3((7, 7, 7))
    b.crse_lo, b.crse_hi = cb._i3((0, 0, 0)), cb._i3((3, 3, 3))
    b.reg_lo, b.reg_hi = cb._i3((0, 0, 0)), cb._i3((3, 3, 3))
    return b


def _create(groups):
    arr = (cb.CxRestrictGroup * len(groups))(*groups)
    res = (ctypes.c_int * len(groups))(*([-1] * len(groups)))
    h = ctypes.c_void_p()
    rc = cb.lib().cx_restrict_groups_plan_create(arr, len(groups), res, ctypes.byref(h))
    return rc, list(res), h


def test_groups_plan_rejects_bad_groups():
    fabs = (cb.CxRestrictBox * 2)(_box(7, 2), _box(7, 3))
    ptr = ctypes.cast(fabs, ctypes.POINTER(cb.CxRestrictBox))
    # a FAB pair whose ncomp is not the group's (time level 1 of 2 is not
    # restricted, so this is time level 0's second pair)
    g = cb.CxRestrictGroup(7, 2, 1, 1, 0, 2, ptr)
    rc, res, h = _create([g])
    assert rc == cb.CX_EINVAL and res == [0] and not h.value
    assert b"ncomp differs" in cb.lib().cx_last_error()
    g = cb.CxRestrictGroup(9, 2, 1, 1, 0, 1, ptr)
    rc, res, h = _create([g])
    assert rc == cb.CX_EINVAL and not h.value
    g = cb.CxRestrictGroup(7, 2, 2, 1, 0, 1, None)
    rc, res, h = _create([g])
    assert rc == cb.CX_EINVAL and not h.value


def test_groups_plan_skipped_groups_need_no_fabs():
    # only skipped groups: nothing to restrict, a valid empty selection (the
    # plan itself needs a device)
    g1 = cb.CxRestrictGroup(7, 2, 3, 0, 0, 0, None)
    g2 = cb.CxRestrictGroup(0, 1, 1, 1, 1, 0, None)
    rc, res, h = _create([g1, g2])
    assert res == [0, 0]
    assert rc in (cb.CX_OK, cb.CX_ENODEVICE)
    if rc == cb.CX_OK:
        cb.lib().cx_restrict_plan_destroy(h)
