"""Autotuner of the separable prolongation kernels.

Every separable operator runs on one streaming-kernel instantiation per
stencil pair and centring.  Each instantiation has a schedule (0: two CTAs
per SM with the x-pass task loop unrolled; 1: three CTAs per SM with a
smaller, rolled loop body) and a cap on the fine z points of a work item (the
z chunk; whole columns up to the cap).  Which is faster depends on the pair,
the centring and the box sizes, so this script measures it.

For every instantiation the tuning workloads use, it times each candidate
(schedule 0/1 x cap 128/64/32) with the other instantiations at their best so
far, on the level plan of every workload that contains it, scores the sum of
the step times relative to the untuned schedule (0, cap 128), keeps the best
and moves on (one coordinate-descent round, instantiations in order of the
fine points they serve).  It then writes the table the library reads at plan
creation, csrc/stream_tuned.h; rebuild (python -m carpetx_b200.build) to use
it.  Results do not depend on the schedule, only the time does.

The workloads are seeded synthetic levels of the benchmark configurations:
the mixed 512-box level (24 variables), the shock level's minmod transfer
(64 boxes of 64^3 cells, 5 variables), the differentiated configuration's
forward level (64 boxes, 4 variables) and the conservative 128^3-cell box
(8 variables).

    python -m carpetx_b200.tune [--steps 10] [--out PATH] [--dry-run]
"""
import argparse
import datetime
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "stream_tuned.h")
NKINDS = 136
# stream_pairs.h, in order (pair index I -> vertex kind / cell kind)
PAIRS = ["VcPoly<1>/CcPoly<1>", "VcPoly<3>/CcPoly<3>", "VcPoly<5>/CcPoly<5>",
         "VcPoly<7>/CcPoly<7>", "VcCons<0>/CcCons<0>", "VcCons<1>/CcCons<2>",
         "VcPoly<1>/CcCons<0>", "VcPoly<3>/CcCons<2>", "VcPoly<5>/CcCons<4>",
         "VcPoly<7>/CcCons<6>", "VcPoly<1>/CcMinmod", "VcPoly<3>/CcMinmod",
         "VcPoly<5>/CcMinmod", "VcPoly<1>/CcCons<1>", "VcPoly<3>/CcCons<3>",
         "VcPoly<5>/CcCons<5>", "VcPoly<7>/CcCons<7>"]
CANDIDATES = [(s, z) for s in (0, 1) for z in (128, 64, 32)]
UNTUNED = (0, 128)


def kind_name(k):
    cm = k % 8
    cent = "".join("C" if (cm >> (2 - d)) & 1 else "V" for d in range(3))
    return f"{PAIRS[k // 8]} {cent}"


def _shape(lo, hi):
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


def workloads(cb, torch, dev, seed=2026):
    """(name, list of LevelPlan box dicts) of the tuning workloads, data on
    the device."""
    from carpetx_b200.workloads import mixed_level_boxes, shock_level_boxes
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    def fab(ncomp, lo, hi):
        return torch.randn((ncomp,) + _shape(lo, hi), dtype=torch.float64, device=dev,
                           generator=gen)

    def box(op, n, clo, chi, flo, fhi):
        return dict(op=op, ncomp=n, crse=fab(n, clo, chi), crse_lo=clo, crse_hi=chi,
                    fine=torch.empty((n,) + _shape(flo, fhi), dtype=torch.float64, device=dev),
                    fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi)

    out = []
    lvl = []
    for it, clo, chi, flo, fhi in mixed_level_boxes(seed, nboxes=512):
        typ, order = ("interpolate", 5) if it == 0 else ("hermite", 3)
        lvl.append(box(cb.Op(typ, order, it), 24, clo, chi, flo, fhi))
    out.append(("level512", lvl))
    mm = cb.Op("minmod", 1, 7)
    out.append(("shock_minmod", [box(mm, 5, clo, chi, flo, fhi)
                                 for _, clo, chi, flo, fhi in shock_level_boxes()]))
    rng = np.random.default_rng(seed + 5)
    diff = []
    for i in range(64):
        n = np.round(np.exp(rng.uniform(np.log(32), np.log(96), 3))).astype(int)
        typ, order, it = ("interpolate", 5, 0) if i % 2 == 0 else ("conservative", 1, 7)
        cc = 1 if it == 7 else 0
        flo = (0, 0, 0)
        fhi = tuple(int(2 * n[d] - 1 - (1 - cc)) for d in range(3))
        op = cb.Op(typ, order, it)
        clo, chi = op.coarse_box(flo, fhi)
        diff.append(box(op, 4, clo, chi, flo, fhi))
    out.append(("differentiated_forward", diff))
    cons = cb.Op("conservative", 1, 7)
    out.append(("conservative128", [box(cons, 8, (-3, -3, -3), (130, 130, 130), (0, 0, 0),
                                        (255, 255, 255))]))
    return out


def time_plan(cb, torch, boxes, steps):
    plan = cb.LevelPlan(boxes)
    for _ in range(2):
        plan.execute()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        plan.execute()
    e1.record()
    torch.cuda.synchronize()
    plan.close()
    return e0.elapsed_time(e1) / steps


def tune(steps=10, out=OUT, dry_run=False):
    import torch
    import carpetx_b200 as cb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    L = cb.lib()
    wls = workloads(cb, torch, dev)
    # fine points per instantiation and the workloads it appears in
    weight, where = {}, {}
    for w, (name, boxes) in enumerate(wls):
        for b in boxes:
            k = L.cx_debug_stream_kind(b["op"].handle)
            if k < 0:
                continue
            pts = b["ncomp"] * int(np.prod(_shape(b["fine_lo"], b["fine_hi"])))
            weight[k] = weight.get(k, 0) + pts
            where.setdefault(k, set()).add(w)
    kinds = sorted(weight, key=lambda k: -weight[k])

    def setk(k, cand):
        if L.cx_debug_set_stream_schedule(k, cand[0], cand[1]) != cb.CX_OK:
            raise RuntimeError(L.cx_last_error().decode())

    # untuned reference times
    for k in kinds:
        setk(k, UNTUNED)
    base = {w: time_plan(cb, torch, wls[w][1], steps) for w in range(len(wls))}
    best = {k: UNTUNED for k in kinds}
    log = {}
    for k in kinds:
        res = {}
        for cand in CANDIDATES:
            setk(k, cand)
            res[cand] = sum(time_plan(cb, torch, wls[w][1], steps) / base[w] for w in where[k])
        best[k] = min(res, key=res.get)
        setk(k, best[k])
        log[k] = {f"{s}/{z}": round(v, 4) for (s, z), v in res.items()}
        print(f"{kind_name(k):28s} best schedule {best[k][0]} cap {best[k][1]}  "
              f"(relative step time {res[best[k]]:.4f} vs {res[UNTUNED]:.4f} untuned)",
              flush=True)
    tuned = {w: time_plan(cb, torch, wls[w][1], steps) for w in range(len(wls))}
    L.cx_debug_set_stream_schedule(-1, -1, 0)
    summary = {wls[w][0]: {"untuned_ms": round(base[w], 4), "tuned_ms": round(tuned[w], 4)}
               for w in range(len(wls))}
    print(json.dumps(summary))
    if not dry_run:
        write_table(out, best, log, summary, torch.cuda.get_device_name(0))
    return best, summary


def write_table(path, best, log, summary, gpu):
    entries = []
    for k in range(NKINDS):
        s, z = best.get(k, (-1, 0))
        entries.append(f"{{{s}, {z}}}")
    lines = ["// Tuned schedule and z-chunk cap per streaming-kernel instantiation",
             "// (8 x stencil pair + centring, stream_pairs.h): sched -1 and maxz 0 mean",
             "// not tuned (the default rule of stream_sched / a cap of 128).  Written by",
             f"// carpetx_b200/tune.py on {gpu}, {datetime.date.today().isoformat()}.",
             "// Per tuned instantiation, the relative step time of each candidate",
             "// (schedule/cap) summed over the tuning workloads that contain it:"]
    for k in sorted(log):
        lines.append(f"//   {k:3d} {kind_name(k)}: " +
                     ", ".join(f"{c} {v}" for c, v in log[k].items()))
    lines.append("// Level step times, untuned (schedule 0, cap 128) and tuned, ms:")
    for name, v in summary.items():
        lines.append(f"//   {name}: {v['untuned_ms']} -> {v['tuned_ms']}")
    lines += ["#pragma once", "", "namespace cxb {", "struct StreamTuned {",
              "  signed char sched;", "  short maxz;", "};",
              f"constexpr StreamTuned kStreamTuned[{NKINDS}] = {{"]
    for i in range(0, NKINDS, 8):
        lines.append("    " + ", ".join(entries[i:i + 8]) + ",")
    lines += ["};", "} // namespace cxb", ""]
    with open(path, "w") as f:
        f.write("\n".join(lines))
    print(f"wrote {path}")


if __name__ == "__main__":
    p = argparse.ArgumentParser()
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--out", default=OUT)
    p.add_argument("--dry-run", action="store_true")
    a = p.parse_args()
    if HERE not in sys.path:
        sys.path.insert(0, os.path.dirname(HERE))
    tune(a.steps, a.out, a.dry_run)
