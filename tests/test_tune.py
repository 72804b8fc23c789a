"""Host side of the streaming kernels' tuning: the instantiation index of an
operator, the schedule settings' argument checks and the tuner's table
writer (no device work)."""
import re

import carpetx_b200 as cb
from carpetx_b200 import tune


def test_stream_kind_of_operators():
    L = cb.lib()
    # interpolate o5 VVV: pair 2 (VcPoly<5>/CcPoly<5>), centring 0
    assert L.cx_debug_stream_kind(cb.Op("interpolate", 5, 0).handle) == 8 * 2 + 0
    # hermite o3 VCC: pair 14 (VcPoly<3>/CcCons<3>), centring 3
    assert L.cx_debug_stream_kind(cb.Op("hermite", 3, 3).handle) == 8 * 14 + 3
    assert tune.kind_name(8 * 14 + 3) == "VcPoly<3>/CcCons<3> VCC"
    # ENO is not served by the streaming kernels
    assert L.cx_debug_stream_kind(cb.Op("eno", 3, 7).handle) == -1


def test_schedule_settings_are_checked():
    L = cb.lib()
    try:
        for args in [(136, 0, 0), (-2, 0, 0), (0, 2, 0), (0, 0, 130), (0, 0, 15), (0, 0, 33)]:
            assert L.cx_debug_set_stream_schedule(*args) == cb.CX_EINVAL, args
        for args in [(5, 1, 64), (-1, 0, 128), (-1, -1, 0)]:
            assert L.cx_debug_set_stream_schedule(*args) == cb.CX_OK, args
    finally:
        L.cx_debug_set_stream_schedule(-1, -1, 0)


def test_table_writer(tmp_path):
    p = tmp_path / "t.h"
    best = {16: (0, 128), 115: (1, 64)}
    log = {16: {"0/128": 1.0}, 115: {"1/64": 0.97}}
    tune.write_table(str(p), best, log, {"level512": {"untuned_ms": 5.0, "tuned_ms": 4.9}}, "GPU")
    s = p.read_text()
    entries = re.findall(r"\{(-?\d+), (\d+)\}", s.split("kStreamTuned")[1])
    assert len(entries) == 136
    assert entries[16] == ("0", "128") and entries[115] == ("1", "64")
    assert entries[0] == ("-1", "0")
