"""Benchmark of the batched level prolongation (FP64 fine points per second).

Workload (default, "level512"): one refinement level of 512 boxes, coarse cells
per direction round(exp(U[ln 8, ln 64])) (seeded), 3 ghost zones, 24 FP64
variables per var (per-component transfers), centrings uniform over VVV, CCC,
VVC, VCC; VVV boxes use "interpolate" order 5, the staggered ones "hermite"
order 3.  Synthetic data (seeded normal values; the operators are linear, the
values do not change the work).

With N ranks (one per GPU, launched by torchrun) the level has 512 x N boxes,
distributed over the ranks by the knapsack mapping of
carpetx_b200.distribute; every rank transfers the boxes it owns (weak
scaling, no data-path collective) and the time is the slowest rank's.

One step = prolongation of every box and component of the level.  Reported:
  value      fine points/s of the batched transfer (one persistent launch,
             replayed from a CUDA graph), inputs resident in HBM
  per_box    the same work launched once per box per component (the
             reference's launch granularity), our kernel
  e2e        through the C ABI with host buffers: pinned host -> device copy
             of the coarse data, the level transfer, device -> host copy of
             the fine data, every step; the level in 8 box batches (one plan
             each) so that copies in, transfers and copies out overlap
  roofline   algorithmic bytes 8 (|CoarseBox(region)| + |region|) per box and
             component over the kernel time, against the measured HBM copy
             bandwidth
  adjoint    forward and adjoint (P^T) time per pass of the differentiated
             configuration (64 boxes, 32-96 coarse points per direction, 4
             variables), as level plans and one launch per box, and the
             adjoint/forward ratios
  restriction  average_down of the conservative configuration (256^3 ->
             128^3, 8 variables): time, GB/s and fraction of the HBM peak
  limited    ENO order 3 and minmod (CCC, 64 boxes of 64^3 coarse cells, 5
             variables) as level plans: fine points/s
  halo       same-level halo exchange (FillBoundary) of the boundary leg's
             level: every ghost point inside the domain from its neighbour,
             one copy-plan launch per step (L2 flushed between steps)
  boundary   outer boundary conditions of a level (the step after a
             prolongation): a 256^3-cell domain in 512 FABs of 32^3 cells, 3
             ghosts, 16 variables, reflection / Dirichlet / linear
             extrapolation / Robin / Neumann faces; one plan launch per step
             (L2 flushed between steps), one launch per FAB beside it, and the
             reference's BoundaryCondition on the host over the same FABs
  cpu_baseline  the reference operators compiled for the host
             (oracle/_ref, all host threads, OpenMP over boxes) on one
             component of every box

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 fine points/s, batched persistent level prolongation"
UNIT = "fine points/s"
L2_BYTES = 126 * 1024 * 1024
E2E_BATCHES = 8  # box batches of the end-to-end leg's copy/transfer pipeline
E2E_CHUNK_MB = 0  # largest single copy of that pipeline, MB (0: one copy per batch)
# ncu DRAM bytes per fine point of the level512 workload's step (the eight
# separable kernels), from a capture of the same 512 boxes with 2 components
# instead of 24 (1/12 of the fine points) with --cache-control none, so that
# write-backs of lines a launch dirtied count in the launches that follow:
# 579,898,112 B read + 2,769,938,688 B written over 16 launches (two steps)
# for 172,696,778 fine points per step; the traffic grows with the fine points
TRAFFIC_PER_FINE_POINT = (579898112 + 2769938688) / 2 / 172696778


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="level512", choices=["level512", "cons128"])
    p.add_argument("--seed", type=int, default=2026)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--per-box-steps", type=int, default=2)
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--e2e-batches", type=int, default=E2E_BATCHES,
                   help="e2e: batches of consecutive boxes, one plan each")
    p.add_argument("--e2e-chunk-mb", type=int, default=E2E_CHUNK_MB,
                   help="e2e: largest single host <-> device copy, MB (0: one per batch)")
    p.add_argument("--adjoint-steps", type=int, default=3,
                   help="passes of the forward/adjoint comparison (0: skip)")
    p.add_argument("--adjoint-boxes", type=int, default=64,
                   help="boxes of the adjoint leg's level (64: the differentiated configuration)")
    p.add_argument("--adjoint-batch", type=int, default=16,
                   help="levels of the adjoint leg's streamed batch (0: skip the batch)")
    p.add_argument("--restrict-steps", type=int, default=5,
                   help="passes of the restriction leg (0: skip)")
    p.add_argument("--limited-steps", type=int, default=2,
                   help="passes of the ENO / minmod leg (0: skip)")
    p.add_argument("--limited-boxes", type=int, default=64,
                   help="boxes of the shock level the ENO / minmod leg takes (at most 64)")
    p.add_argument("--halo-steps", type=int, default=5,
                   help="executions of the halo-exchange leg (0: skip)")
    p.add_argument("--boundary-steps", type=int, default=5,
                   help="executions of the boundary-condition leg (0: skip)")
    p.add_argument("--sync-steps", type=int, default=10,
                   help="ghost-shell and sync-chain steps (0: skip)")
    p.add_argument("--tune-steps", type=int, default=5,
                   help="steps of the tuned / untuned schedule comparison (0: skip)")
    p.add_argument("--boxes", type=int, default=512, help="level512: number of boxes")
    p.add_argument("--ncomp", type=int, default=24, help="level512: variables per box")
    return p.parse_args()


def box_shape(lo, hi):
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


def npts(lo, hi):
    return int(np.prod(box_shape(lo, hi)))


def workload(name, seed, nboxes=512, ncomp=24):
    """List of boxes (type, order, indextype, crse_lo, crse_hi, fine_lo, fine_hi,
    ncomp) and a description."""
    from carpetx_b200.workloads import mixed_level_boxes
    if name == "level512":
        out = []
        for it, clo, chi, flo, fhi in mixed_level_boxes(seed, nboxes=nboxes):
            typ, order = ("interpolate", 5) if it == 0 else ("hermite", 3)
            out.append((typ, order, it, clo, chi, flo, fhi, ncomp))
        return out, {"workload": f"level512: {nboxes} boxes, coarse 8-64 cells/dim log-uniform, "
                                 f"3 ghosts, {ncomp} vars per var, VVV interpolate o5 / "
                                 "VVC,VCC,CCC hermite o3",
                     "boxes": nboxes, "ncomp": ncomp}
    # one 128^3-cell box, 3 ghosts, 8 vars, conservative order 1 (CC CONS 2)
    return ([("conservative", 1, 7, (-3, -3, -3), (130, 130, 130), (0, 0, 0), (255, 255, 255), 8)],
            {"workload": "cons128: conservative o1 CCC, 128^3 -> 256^3 cells, 3 ghosts, 8 vars",
             "boxes": 1, "ncomp": 8})


def adjoint_leg(args, cb, torch, dev, max_over_ranks, barrier):
    """Forward and adjoint (P^T, cx_prolong_adjoint_box) of the differentiated
    configuration, one launch per box each: 64 boxes with coarse points per
    direction round(exp(U[ln 32, ln 96])), 4 components, alternately
    interpolate order 5 VVV and conservative order 1 CCC, fine region = the
    refined box.  Returns the per-pass times and their ratio."""
    rng = np.random.default_rng(args.seed + 5)
    boxes = []
    for i in range(64):
        n = np.round(np.exp(rng.uniform(np.log(32), np.log(96), 3))).astype(int)
        if i >= args.adjoint_boxes:
            continue
        typ, order, it = ("interpolate", 5, 0) if i % 2 == 0 else ("conservative", 1, 7)
        cc = 1 if it == 7 else 0
        flo = (0, 0, 0)
        fhi = tuple(int(2 * n[d] - 1 - (1 - cc)) for d in range(3))
        op = cb.Op(typ, order, it)
        clo, chi = op.coarse_box(flo, fhi)
        boxes.append((op, clo, chi, flo, fhi))
    nc = 4
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 5)
    data = []
    for op, clo, chi, flo, fhi in boxes:
        u = torch.randn((nc,) + box_shape(clo, chi), dtype=torch.float64, device=dev, generator=gen)
        f = torch.empty((nc,) + box_shape(flo, fhi), dtype=torch.float64, device=dev)
        ub = torch.empty_like(u)
        data.append((op, u, clo, chi, f, flo, fhi, ub))
    nfine = sum(nc * npts(b[5], b[6]) for b in data)

    def fwd():
        for op, u, clo, chi, f, flo, fhi, ub in data:
            cb.prolong_box(op, u, clo, chi, f, flo, fhi, flo, fhi, nc)

    def adj():
        for op, u, clo, chi, f, flo, fhi, ub in data:
            cb.prolong_adjoint_box(op, u, clo, chi, f, flo, fhi, flo, fhi, nc, ub)

    def plan_boxes(out_crse):
        return [dict(op=op, ncomp=nc, crse=ub if out_crse else u, crse_lo=clo, crse_hi=chi,
                     fine=f, fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi)
                for op, u, clo, chi, f, flo, fhi, ub in data]

    plan_f = cb.LevelPlan(plan_boxes(False))
    plan_a = cb.LevelPlan(plan_boxes(True), adjoint=True)
    out = {"workload": f"{len(boxes)} boxes, coarse 32-96 points/dim log-uniform, 4 vars, interpolate o5 VVV "
                       "/ conservative o1 CCC; level plans (one persistent launch per stencil "
                       "pair) and one launch per box",
           "fine_points": nfine}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, fn in (("fwd_level", plan_f.execute), ("adj_level", plan_a.execute),
                     ("fwd_per_box", fwd), ("adj_per_box", adj)):
        for _ in range(2):
            fn()
        barrier()
        e0.record()
        for _ in range(args.adjoint_steps):
            fn()
        e1.record()
        barrier()
        out[name + "_ms"] = max_over_ranks(e0.elapsed_time(e1)) / args.adjoint_steps
    out["adj_over_fwd"] = out["adj_level_ms"] / out["fwd_level_ms"]
    out["adj_over_fwd_per_box"] = out["adj_per_box_ms"] / out["fwd_per_box_ms"]
    out["adj_level_gbs"] = plan_a.stats()["bytes"] / (out["adj_level_ms"] / 1e3) / 1e9
    plan_f.close()
    plan_a.close()
    del data
    if args.adjoint_batch > 0:
        out["batch16"] = adjoint_batch(args, cb, torch, dev, max_over_ranks, barrier, nc,
                                       args.adjoint_batch)
    return out


def adjoint_batch(args, cb, torch, dev, max_over_ranks, barrier, nc, nlevels=16):
    """The differentiated configuration as stated: a batch of 16 independent
    levels of 64 boxes each (coarse points per direction log-uniform in
    [32, 96], interpolate o5 VVV / conservative o1 CCC alternately, 4
    variables), streamed level by level: every level's boxes are views into
    one set of buffers sized for the largest level, so the batch needs one
    level's memory.  One step = the forward (or the adjoint) of all 16
    levels, one plan execution per level; plans are built before timing."""
    levels = []
    for lv in range(nlevels):
        rng = np.random.default_rng(args.seed + 5 + 1000 * (lv + 1))
        bl = []
        for i in range(64):
            n = np.round(np.exp(rng.uniform(np.log(32), np.log(96), 3))).astype(int)
            typ, order, it = ("interpolate", 5, 0) if i % 2 == 0 else ("conservative", 1, 7)
            cc = 1 if it == 7 else 0
            flo = (0, 0, 0)
            fhi = tuple(int(2 * n[d] - 1 - (1 - cc)) for d in range(3))
            op = cb.Op(typ, order, it)
            clo, chi = op.coarse_box(flo, fhi)
            bl.append((op, clo, chi, flo, fhi))
        levels.append(bl)
    csz = max(sum(nc * npts(b[1], b[2]) for b in bl) for bl in levels)
    fsz = max(sum(nc * npts(b[3], b[4]) for b in bl) for bl in levels)
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 6)
    u = torch.randn(csz, dtype=torch.float64, device=dev, generator=gen)
    ub = torch.empty(csz, dtype=torch.float64, device=dev)
    f = torch.randn(fsz, dtype=torch.float64, device=dev, generator=gen)
    plans_f, plans_a, nfine = [], [], 0
    for bl in levels:
        fb, ab, co, fo = [], [], 0, 0
        for op, clo, chi, flo, fhi in bl:
            cs, fs = nc * npts(clo, chi), nc * npts(flo, fhi)
            cv = u[co:co + cs].view((nc,) + box_shape(clo, chi))
            bv = ub[co:co + cs].view((nc,) + box_shape(clo, chi))
            fv = f[fo:fo + fs].view((nc,) + box_shape(flo, fhi))
            fb.append(dict(op=op, ncomp=nc, crse=cv, crse_lo=clo, crse_hi=chi, fine=fv,
                           fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi))
            ab.append(dict(fb[-1], crse=bv))
            co += cs
            fo += fs
            nfine += fs
        plans_f.append(cb.LevelPlan(fb))
        plans_a.append(cb.LevelPlan(ab, adjoint=True))
    res = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for name, plans in (("fwd", plans_f), ("adj", plans_a)):
        for p in plans:
            p.execute()
        barrier()
        e0.record()
        for _ in range(max(1, args.adjoint_steps // 2)):
            for p in plans:
                p.execute()
        e1.record()
        barrier()
        res[name] = max_over_ranks(e0.elapsed_time(e1)) / max(1, args.adjoint_steps // 2)
    for p in plans_f + plans_a:
        p.close()
    return {"workload": f"{nlevels} independent levels of 64 boxes, coarse 32-96 points/dim "
                        f"log-uniform, {nc} vars, interpolate o5 VVV / conservative o1 CCC, "
                        "streamed level by level through one level's buffers",
            "levels": nlevels, "fine_points": nfine, "buffer_gb": 8 * (2 * csz + fsz) / 1e9,
            "fwd_ms": res["fwd"], "adj_ms": res["adj"], "adj_over_fwd": res["adj"] / res["fwd"]}


def restrict_leg(args, cb, torch, dev, max_over_ranks, barrier, peak):
    """Restriction of the conservative configuration (cx_restrict_box): CCC
    mean of the 2x2x2 children, fine cells 0..255 -> coarse region 0..127 of
    the coarse box -3..130 (3 ghosts), 8 components.  Algorithmic bytes: 8 per
    fine point read + 8 per coarse point written."""
    nc = 8
    flo, fhi = (0, 0, 0), (255, 255, 255)
    clo, chi = (-3, -3, -3), (130, 130, 130)
    rlo, rhi = (0, 0, 0), (127, 127, 127)
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 2)
    f = torch.randn((nc,) + box_shape(flo, fhi), dtype=torch.float64, device=dev, generator=gen)
    c = torch.zeros((nc,) + box_shape(clo, chi), dtype=torch.float64, device=dev)
    nbytes = 8 * nc * (npts(flo, fhi) + npts(rlo, rhi))

    def step():
        cb.restrict_box(7, f, flo, fhi, c, clo, chi, rlo, rhi, nc)

    for _ in range(3):
        step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.restrict_steps):
        step()
    e1.record()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1)) / args.restrict_steps
    gbs = nbytes / (ms / 1e3) / 1e9
    del f, c
    out = {"workload": "restriction CCC (average_down), fine 256^3 -> coarse 128^3, 8 vars, "
                       "one launch", "ms": ms, "bytes": nbytes, "achieved_gbs": gbs,
           "frac_of_peak": gbs / peak}
    # the whole mixed level (the prolongation's 512 boxes, four centrings, 8
    # vars) restricted by one plan (one launch per index type) and by one
    # cx_restrict_box call per box
    from carpetx_b200.workloads import mixed_level_boxes
    boxes = []
    for it, clo, chi, flo, fhi in mixed_level_boxes(args.seed, nboxes=512):
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        fine = torch.empty((nc,) + box_shape(flo, fhi), dtype=torch.float64, device=dev)
        fine.normal_(generator=gen)
        crse = torch.zeros((nc,) + box_shape(clo, chi), dtype=torch.float64, device=dev)
        boxes.append(dict(indextype=it, ncomp=nc, fine=fine, fine_lo=flo, fine_hi=fhi, crse=crse,
                          crse_lo=clo, crse_hi=chi, reg_lo=tuple(v // 2 for v in flo),
                          reg_hi=tuple((fhi[d] - cc[d]) // 2 for d in range(3))))
    plan = cb.RestrictPlan(boxes)
    st = plan.stats()

    def per_box():
        for b in boxes:
            cb.restrict_box(b["indextype"], b["fine"], b["fine_lo"], b["fine_hi"], b["crse"],
                            b["crse_lo"], b["crse_hi"], b["reg_lo"], b["reg_hi"], nc)

    res = {}
    for name, fn in (("plan", plan.execute), ("per_box", per_box)):
        for _ in range(3):
            fn()
        barrier()
        e0.record()
        for _ in range(args.restrict_steps):
            fn()
        e1.record()
        barrier()
        res[name] = max_over_ranks(e0.elapsed_time(e1)) / args.restrict_steps
    lgbs = st["bytes"] / (res["plan"] / 1e3) / 1e9
    out["level"] = {"workload": f"{len(boxes)} boxes of the mixed level (VVV, CCC, VVC, VCC), "
                                f"{nc} vars; inputs {sum(b['fine'].numel() for b in boxes) * 8 / 1e9:.1f}"
                                " GB > L2, no flush",
                    "ms": res["plan"], "launches": st["launches"], "bytes": st["bytes"],
                    "achieved_gbs": lgbs, "frac_of_peak": lgbs / peak,
                    "per_box_ms": res["per_box"], "per_box_launches": len(boxes),
                    "batched_speedup": res["per_box"] / res["plan"]}
    plan.close()
    del boxes
    return out


def limited_leg(args, cb, torch, dev, max_over_ranks, barrier):
    """Limited operators of the shock configuration: ENO order 3 and minmod,
    all directions cell centred, 64 boxes of 64^3 coarse cells (3 ghosts)
    tiling a 256^3-cell cube, 5 variables (rho, momenta, E) of the seeded
    shock state of carpetx_b200.workloads.shock_state: a planar shock with a
    random normal, 10x density and pressure jumps, Gaussian blobs and 1e-6
    noise.  A level plan each; the data is generated on the host once."""
    from carpetx_b200.workloads import shock_fab, shock_level_boxes, shock_state
    nc = 5
    state = shock_state(args.seed + 4, 256)
    sboxes = shock_level_boxes()[:max(1, args.limited_boxes)]
    nb = len(sboxes)
    flo0, fhi0 = sboxes[0][3], sboxes[0][4]
    out = {"workload": f"{nb} boxes, 64^3 coarse cells -> 128^3 fine, {nc} vars (rho, momenta, "
                       "E) of a planar shock (random normal, 10x rho and p jumps) with Gaussian "
                       "blobs and 1e-6 noise, CCC; level plans",
           "fine_points": nb * nc * npts(flo0, fhi0)}
    crse = [torch.from_numpy(shock_fab(state, clo, chi, bid)).to(dev)
            for bid, clo, chi, flo, fhi in sboxes]
    fine = [torch.empty((nc,) + box_shape(flo, fhi), dtype=torch.float64, device=dev)
            for bid, clo, chi, flo, fhi in sboxes]
    L = cb.lib()
    for typ, order, untuned in (("eno", 3, False), ("minmod", 1, False), ("minmod", 1, True)):
        op = cb.Op(typ, order, 7)
        boxes = [dict(op=op, ncomp=nc, crse=c, crse_lo=clo, crse_hi=chi, fine=f, fine_lo=flo,
                      fine_hi=fhi, reg_lo=flo, reg_hi=fhi)
                 for (bid, clo, chi, flo, fhi), c, f in zip(sboxes, crse, fine)]
        if untuned:
            # the plan as the untuned schedule builds it (every instantiation
            # schedule 0, cap 128), against the tuned table
            L.cx_debug_set_stream_schedule(-1, 0, 128)
            plan = cb.LevelPlan(boxes)
            L.cx_debug_set_stream_schedule(-1, -1, 0)
            typ = "minmod_untuned"
        else:
            plan = cb.LevelPlan(boxes)
        for _ in range(2):
            plan.execute()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.limited_steps):
            plan.execute()
        e1.record()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1)) / args.limited_steps
        out[f"{typ}_ms"] = ms
        out[f"{typ}_pts_per_s"] = out["fine_points"] / (ms / 1e3)
        out[f"{typ}_launches"] = plan.stats()["launches"]
        plan.close()
        if not untuned:
            # the adjoint level plan, linearised at the same coarse data
            # (decision pass and gather per box): P^T of the fine data
            cbar = [torch.empty_like(c) for c in crse]
            aplan = cb.LevelPlan([dict(b, crse=cb_, crse_at=b["crse"])
                                  for b, cb_ in zip(boxes, cbar)], adjoint=True)
            aplan.execute()
            barrier()
            e0.record()
            for _ in range(args.limited_steps):
                aplan.execute()
            e1.record()
            barrier()
            ms_a = max_over_ranks(e0.elapsed_time(e1)) / args.limited_steps
            out[f"{typ}_adjoint_ms"] = ms_a
            out[f"{typ}_adjoint_over_forward"] = ms_a / ms
            aplan.close()
            del cbar
        del boxes
    return out


def sync_leg(args, cb, torch, dev, max_over_ranks, barrier, peak):
    """The per-step sync's prolongation on ghost shells, and the whole sync.

    ghost_shell: every box of the mixed 512-box level as a fine FAB with 3
    ghost cells per side whose whole shell is uncovered (the boxes do not
    touch), 24 variables, the level512 operators; the shell is the FAB minus
    its valid box, six slabs 3 fine points deep, prolongated from the box's
    coarse FAB through one level plan, against one launch per slab.

    sync_chain: the six steps of carpetx_b200.sync.SyncChain (FillBoundary,
    coarse-patch gather, coarse boundary conditions, prolongation of the
    fine patches, scatter, fine boundary conditions) on a cell-centred coarse
    level of 128^3 cells in 64 FABs of 32^3 and a fine level over its lower
    corner octant, 256^3 ... 128^3 fine cells in 64 FABs of 32^3, 3 ghosts,
    16 variables (the boundary conditions take at most 16), hermite order 3;
    replayed as one CUDA graph."""
    from carpetx_b200.sync import SyncChain, subtract, tiled_fabs
    from carpetx_b200.workloads import boundary_spec, mixed_level_boxes
    out = {}
    nc, ng = args.ncomp, 3
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 7)
    # ghost shells of the level512 boxes
    recs, ctot, ftot = [], 0, 0
    for it, clo0, chi0, flo, fhi in mixed_level_boxes(args.seed, nboxes=args.boxes):
        typ, order = ("interpolate", 5) if it == 0 else ("hermite", 3)
        op = cb.Op(typ, order, it)
        glo = tuple(flo[d] - ng for d in range(3))
        ghi = tuple(fhi[d] + ng for d in range(3))
        clo, chi = op.coarse_box(glo, ghi)
        recs.append((op, clo, chi, glo, ghi, subtract((glo, ghi), (flo, fhi)), ctot, ftot))
        ctot += nc * npts(clo, chi)
        ftot += nc * npts(glo, ghi)
    crse = torch.empty(ctot, dtype=torch.float64, device=dev)
    crse.normal_(generator=gen)
    fine = torch.zeros(ftot, dtype=torch.float64, device=dev)
    boxes, calls = [], []
    L = cb.lib()
    I3 = ctypes.c_int * 3
    stream = torch.cuda.Stream(device=dev)
    sp = ctypes.c_void_p(stream.cuda_stream)
    shell_pts = 0
    for op, clo, chi, glo, ghi, slabs, co, fo in recs:
        c = crse[co:co + nc * npts(clo, chi)].view((nc,) + box_shape(clo, chi))
        f = fine[fo:fo + nc * npts(glo, ghi)].view((nc,) + box_shape(glo, ghi))
        for rlo, rhi in slabs:
            boxes.append(dict(op=op, ncomp=nc, crse=c, crse_lo=clo, crse_hi=chi, fine=f,
                              fine_lo=glo, fine_hi=ghi, reg_lo=rlo, reg_hi=rhi))
            calls.append((op.handle, ctypes.c_void_p(c.data_ptr()), I3(*clo), I3(*chi),
                          ctypes.c_void_p(f.data_ptr()), I3(*glo), I3(*ghi), I3(*rlo), I3(*rhi)))
            shell_pts += nc * npts(rlo, rhi)
    plan = cb.LevelPlan(boxes)
    st = plan.stats()

    def timed_graph(fn, steps):
        with torch.cuda.stream(stream):
            fn()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            fn()
        for _ in range(2):
            g.replay()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(steps):
                g.replay()
            e1.record(stream)
        barrier()
        del g
        return max_over_ranks(e0.elapsed_time(e1)) / steps

    def per_slab():
        for c in calls:
            rc = L.cx_prolong_box(*c, nc, 0, sp)
            if rc:
                raise RuntimeError(L.cx_last_error().decode())

    ms = timed_graph(lambda: plan.execute(stream), args.sync_steps)
    ms_pb = timed_graph(per_slab, max(1, args.sync_steps // 5))
    out["ghost_shell"] = {
        "workload": f"{args.boxes} boxes of the mixed level as fine FABs with {ng} ghosts per side, "
                    f"the whole shell uncovered (six slabs {ng} deep per box), {nc} vars, "
                    "interpolate o5 VVV / hermite o3 VVC,VCC,CCC; one level plan, graph replay",
        "regions": len(boxes), "fine_points": shell_pts, "bytes": st["bytes"], "ms": ms,
        "fine_pts_per_s": shell_pts / (ms / 1e3),
        "achieved_gbs": st["bytes"] / (ms / 1e3) / 1e9,
        "frac_of_peak": st["bytes"] / (ms / 1e3) / 1e9 / peak, "launches": st["launches"],
        "per_region_ms": ms_pb, "per_region_launches": len(calls), "batched_speedup": ms_pb / ms}
    plan.close()
    del boxes, calls, crse, fine
    torch.cuda.empty_cache()
    # the whole sync of a refined corner
    nc2 = min(nc, cb.BC_MAX_COMPS)
    op = cb.Op("hermite", 3, 7)
    cfab = tiled_fabs((128, 128, 128), (32, 32, 32), (ng,) * 3)
    ffab = tiled_fabs((128, 128, 128), (32, 32, 32), (ng,) * 3)

    def alloc(fabs):
        out_ = []
        for lo, hi, vlo, vhi in fabs:
            a = torch.full((nc2,) + box_shape(lo, hi), float("nan"), dtype=torch.float64,
                           device=dev)
            sl = tuple(slice(vlo[d] - lo[d], vhi[d] - lo[d] + 1) for d in (2, 1, 0))
            a[(slice(None),) + sl] = torch.rand(a[(slice(None),) + sl].shape, generator=gen,
                                                dtype=torch.float64, device=dev)
            out_.append((a, lo, hi, vlo, vhi))
        return out_

    coarse, finel = alloc(cfab), alloc(ffab)
    faces = [[(0, 4), (0, 2), (0, 4)], [(0, 2), (0, 4), (0, 2)]]
    rng = np.random.default_rng(args.seed + 8)
    cs = boundary_spec(rng, nc2, (1, 1, 1), (128, 128, 128), nghost=ng, faces=faces)
    fs = boundary_spec(rng, nc2, (1, 1, 1), (256, 256, 256), nghost=ng, faces=faces)
    fs["dirichlet"], fs["robin"] = cs["dirichlet"], cs["robin"]
    chain = SyncChain(op, nc2, coarse, finel, (ng,) * 3, cs, fs)
    cst = chain.stats()
    chain_bytes = sum(v["bytes"] for v in cst.values())
    ms_chain = timed_graph(lambda: chain.execute(stream), args.sync_steps)
    steps_ms = {}
    for name, p in chain.steps:
        steps_ms[name] = timed_graph(lambda p=p: p.execute(stream), args.sync_steps)
    # the prolongation writing into the fine FABs (no patch buffers, no scatter)
    fused = SyncChain(op, nc2, coarse, finel, (ng,) * 3, cs, fs, fused=True)
    fst = fused.stats()
    fused_bytes = sum(v["bytes"] for v in fst.values())
    ms_fused = timed_graph(lambda: fused.execute(stream), args.sync_steps)
    fused.close()
    # the coarse level's ghosts synced once (its halo exchange and boundary
    # conditions), then the pieces whose coarse box lies in one coarse FAB
    # read it directly (no gather, no coarse boundary conditions for them)
    cfill = cb.CopyPlan.fill_boundary(coarse, nc2, (ng,) * 3)
    cbcp = cb.BoundaryPlan(cs, [c[:3] for c in coarse])
    with torch.cuda.stream(stream):
        cfill.execute(stream)
        cbcp.execute(stream)
    torch.cuda.synchronize()
    direct = SyncChain(op, nc2, coarse, finel, (ng,) * 3, cs, fs, direct=True)
    dsts = direct.stats()
    direct_bytes = sum(v["bytes"] for v in dsts.values())
    ms_direct = timed_graph(lambda: direct.execute(stream), args.sync_steps)
    ndirect = sum(s is not None for s in direct.src)
    npieces = len(direct.patches)
    direct.close()
    cfill.close()
    cbcp.close()
    out["sync_chain"] = {
        "workload": "FillBoundary, coarse-patch gather, coarse boundary conditions, prolongation "
                    "of the fine patches, scatter, fine boundary conditions: coarse level 128^3 "
                    "cells in 64 FABs of 32^3, fine level over the lower corner octant in 64 "
                    f"FABs of 32^3, {ng} ghosts, {nc2} vars, hermite o3 CCC; one CUDA graph",
        "fine_patches": len(chain.patches), "bytes": chain_bytes, "ms": ms_chain,
        "achieved_gbs": chain_bytes / (ms_chain / 1e3) / 1e9,
        "frac_of_peak": chain_bytes / (ms_chain / 1e3) / 1e9 / peak,
        "steps": {name: {"ms": steps_ms[name], "bytes": cst[name]["bytes"],
                         "frac_of_peak": cst[name]["bytes"] / (steps_ms[name] / 1e3) / 1e9 / peak}
                  for name in steps_ms},
        "fused": {"what": "prolongation into the fine FABs' ghosts, no fine patch buffers or "
                          "scatter (five plans)",
                  "ms": ms_fused, "bytes": fused_bytes,
                  "frac_of_peak": fused_bytes / (ms_fused / 1e3) / 1e9 / peak,
                  "speedup": ms_chain / ms_fused},
        "direct": {"what": "as fused, with the coarse level's ghosts synced: the fine patches, "
                           "cut at the refined coarse FAB faces, whose coarse box lies in one "
                           "coarse FAB read it directly; the rest are gathered",
                   "pieces": npieces, "pieces_direct": ndirect, "ms": ms_direct,
                   "bytes": direct_bytes,
                   "frac_of_peak": direct_bytes / (ms_direct / 1e3) / 1e9 / peak,
                   "speedup": ms_chain / ms_direct}}
    chain.close()
    # reflux of the refined corner's coarse level (CarpetX's Reflux through
    # the FluxRegister): face-centred fluxes on both levels, the same FABs
    def flux_fabs(fabs, d):
        out_ = []
        for a, lo, hi, vlo, vhi in fabs:
            flo, fhi = lo, tuple(v + (e == d) for e, v in enumerate(hi))
            fvhi = tuple(v + (e == d) for e, v in enumerate(vhi))
            t = torch.empty((nc2,) + box_shape(flo, fhi), dtype=torch.float64, device=dev)
            t.normal_(generator=gen)
            out_.append((t, flo, fhi, vlo, fvhi))
        return out_

    cfx = [flux_fabs(coarse, d) for d in range(3)]
    ffx = [flux_fabs(finel, d) for d in range(3)]
    rplan = cb.RefluxPlan(coarse, cfx, ffx, nc2, (1.0 / 128,) * 3)
    rst = rplan.stats()
    ms_r = timed_graph(lambda: rplan.execute(stream), args.sync_steps)
    out["reflux"] = {
        "workload": "the coarse level of the refined corner above: every face of the fine "
                    f"boxes' coarsened boundary with a coarse cell outside, {nc2} vars; "
                    "CrseInit, FineAdd and Reflux fused, one launch per face orientation",
        "faces": rst["faces"], "bytes": rst["bytes"], "launches": rst["launches"], "ms": ms_r,
        "faces_per_s": rst["faces"] * nc2 / (ms_r / 1e3),
        "frac_of_peak": rst["bytes"] / (ms_r / 1e3) / 1e9 / peak}
    rplan.close()
    return out


def boundary_leg(args, cb, torch, dev, max_over_ranks, barrier, peak):
    """Outer boundary conditions of the level of
    carpetx_b200.workloads.BC_LEVEL_FACES (cx_boundary_plan_*): every FAB's
    points outside the domain (1.63 M: neighbouring FABs' ghosts overlap along
    the domain's edges) x 16 variables, per step one launch.
    Algorithmic bytes: 8 written per value, plus 8 read unless Dirichlet.  The
    L2 is flushed (a 256 MiB write) before each timed execution."""
    from carpetx_b200.workloads import BC_LEVEL_FACES, boundary_spec, tiled_level_fabs
    nc, n, g = 16, 256, 3
    spec = boundary_spec(np.random.default_rng(args.seed + 5), nc, (1, 1, 1), (n,) * 3,
                         nghost=g, faces=BC_LEVEL_FACES)
    fabs = tiled_level_fabs((n,) * 3, (32,) * 3, (1, 1, 1), g)
    side = 32 + 2 * g
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 5)
    slab = torch.empty((len(fabs), nc, side, side, side), dtype=torch.float64, device=dev)
    slab.uniform_(-1, 1, generator=gen)
    plan = cb.BoundaryPlan(spec, [(slab[i], lo, hi) for i, (lo, hi) in enumerate(fabs)])
    st = plan.stats()
    flush = torch.empty(256 * 2**20 // 8, dtype=torch.float64, device=dev)
    # FABs that reach outside the domain: the reference builds a
    # BoundaryCondition for these only (driver.cxx:991-994)
    edge = [i for i, (lo, hi) in enumerate(fabs)
            if any(lo[d] < 0 or hi[d] > n - 1 for d in range(3))]
    out = {"workload": f"{len(fabs)} FABs of 32^3 cells (+{g} ghosts) tiling a {n}^3-cell "
                       f"domain, {nc} vars, cell centred; faces x: reflection / Dirichlet, y: "
                       "linear extrapolation / Robin, z: Neumann / linear extrapolation",
           "points": st["points"], "values": st["points"] * nc, "bytes": st["bytes"],
           "fabs_with_boundary": len(edge)}

    def timed(fn, steps):
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total / steps

    for _ in range(3):
        plan.execute()
    barrier()
    ms = max_over_ranks(timed(plan.execute, args.boundary_steps))
    gbs = st["bytes"] / (ms / 1e3) / 1e9
    out.update({"ms": ms, "values_per_s": out["values"] / (ms / 1e3), "achieved_gbs": gbs,
                "frac_of_peak": gbs / peak, "launches_per_step": 1})

    def per_fab():
        for i in edge:
            cb.boundary_box(spec, slab[i], fabs[i][0], fabs[i][1])

    per_fab()
    barrier()
    ms_pf = max_over_ranks(timed(per_fab, max(1, args.boundary_steps // 2)))
    out.update({"per_fab_ms": ms_pf, "per_fab_launches": len(edge),
                "batched_speedup": ms_pf / ms})
    plan.close()
    if not args.no_cpu_baseline:
        from oracle.oracle import RefBoundary
        if RefBoundary.available():
            ref = RefBoundary()
            host = [slab[i].cpu().numpy() for i in edge]
            t0 = time.perf_counter()
            for a, i in zip(host, edge):
                ref.boundary(spec, a, fabs[i][0], fabs[i][1])
            t = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": out["values"] / t, "unit": "values/s", "cores": 1,
                                   "kind": "reference",
                                   "sample": f"BoundaryCondition::apply on all {len(edge)} FABs "
                                             "that reach the boundary (the whole level), one "
                                             "pass; oracle/_ref parity build (-O2, asserts on)"}
    del slab, flush
    return out


def halo_leg(args, cb, torch, dev, max_over_ranks, barrier, peak):
    """FillBoundary (cx_copy_plan_fill_boundary) of a 256^3-cell domain in
    512 FABs of 32^3 cells with 3 ghosts, 16 components, not periodic: each
    FAB's ghost points inside the domain from its neighbours, one launch.
    Algorithmic bytes: 16 per value (one read, one write).  The L2 is
    flushed (a 256 MiB write) before each timed execution."""
    from carpetx_b200.workloads import tiled_level_fabs
    nc, n, g = 16, 256, 3
    fabs = tiled_level_fabs((n,) * 3, (32,) * 3, (1, 1, 1), g)
    side = 32 + 2 * g
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + 6)
    slab = torch.empty((len(fabs), nc, side, side, side), dtype=torch.float64, device=dev)
    slab.uniform_(-1, 1, generator=gen)
    plan = cb.CopyPlan.fill_boundary(
        [(slab[i], lo, hi, tuple(v + g for v in lo), tuple(v - g for v in hi))
         for i, (lo, hi) in enumerate(fabs)], nc, (g, g, g))
    st = plan.stats()
    flush = torch.empty(256 * 2**20 // 8, dtype=torch.float64, device=dev)
    for _ in range(3):
        plan.execute()
    barrier()
    total = 0.0
    for _ in range(args.halo_steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.execute()
        e1.record()
        e1.synchronize()
        total += e0.elapsed_time(e1)
    ms = max_over_ranks(total / args.halo_steps)
    gbs = st["bytes"] / (ms / 1e3) / 1e9
    plan.close()
    del slab, flush
    return {"workload": f"FillBoundary: {len(fabs)} FABs of 32^3 cells (+{g} ghosts) tiling a "
                        f"{n}^3-cell domain, {nc} vars, cell centred, not periodic; one launch",
            "points": st["points"], "pieces": st["pieces"], "values": st["points"] * nc,
            "bytes": st["bytes"], "ms": ms, "values_per_s": st["points"] * nc / (ms / 1e3),
            "achieved_gbs": gbs, "frac_of_peak": gbs / peak, "launches_per_step": 1}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


# --------------------------------------------------------------------------
# CPU baseline: the reference operators compiled for the host

def cpu_lib():
    """(ctypes lib, kind): oracle/_ref (the reference itself) if built, else
    the oracle port."""
    from oracle.oracle import RefOracle, CxOracle
    if RefOracle.available(fast=True):
        L = RefOracle(fast=True).lib
        L.ref_prolong_many.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_void_p),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]
        return L, "reference"
    return CxOracle(), "port"


def cpu_sample(boxes, seed, ncomp_sample=1):
    """Host FABs for one component of every box (the bounded CPU sample)."""
    rng = np.random.default_rng(seed)
    crse, fine = [], []
    for (typ, order, it, clo, chi, flo, fhi, n) in boxes:
        crse.append(rng.standard_normal((ncomp_sample,) + box_shape(clo, chi)))
        fine.append(np.empty((ncomp_sample,) + box_shape(flo, fhi)))
    return crse, fine


def cpu_run(lib, kind, boxes, crse, fine, ncomp_sample=1):
    """One pass of the reference CPU path over the sample; returns seconds."""
    n = len(boxes)
    t0 = time.perf_counter()
    if kind == "reference":
        I = ctypes.c_int
        types = (ctypes.c_char_p * n)(*[b[0].encode() for b in boxes])
        orders = (I * n)(*[b[1] for b in boxes])
        its = (I * n)(*[b[2] for b in boxes])
        cp = (ctypes.c_void_p * n)(*[c.ctypes.data for c in crse])
        fp = (ctypes.c_void_p * n)(*[f.ctypes.data for f in fine])
        flat = lambda k: (I * (3 * n))(*[v for b in boxes for v in b[k]])  # noqa: E731
        nc = (I * n)(*([ncomp_sample] * n))
        t0 = time.perf_counter()
        rc = lib.ref_prolong_many(n, types, orders, its, 0, cp, flat(3), flat(4), fp, flat(5),
                                  flat(6), flat(5), flat(6), nc)
        assert rc == 0
    else:
        for b, c, f in zip(boxes, crse, fine):
            lib.prolong(b[0], b[1], b[2], 0, c, b[3], b[4], f, b[5], b[6], b[5], b[6],
                        ncomp_sample)
    return time.perf_counter() - t0


def cpu_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def cpu_model():
    """The host CPU's model name (as lscpu reports it), from /proc/cpuinfo."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_timed_passes(lib, kind, boxes, crse, fine, min_s=5.0, min_passes=5, max_passes=200):
    """Passes of the reference CPU path over the sample after two warm-up
    passes, until min_s seconds and min_passes passes are reached; returns
    (total seconds, passes)."""
    for _ in range(2):
        cpu_run(lib, kind, boxes, crse, fine)
    t, n = 0.0, 0
    while n < max_passes and (t < min_s or n < min_passes):
        t += cpu_run(lib, kind, boxes, crse, fine)
        n += 1
    return t, n


def run_reference(args, rank):
    """--impl reference: the reference's own CPU implementation of the path on
    the host cores, same workload, one component of every box per step."""
    if rank != 0:
        return
    boxes, cfg = workload(args.workload, args.seed, args.boxes, args.ncomp)
    lib, kind = cpu_lib()
    crse, fine = cpu_sample(boxes, args.seed)
    pts = sum(npts(b[5], b[6]) for b in boxes)
    for _ in range(args.warmup):
        cpu_run(lib, kind, boxes, crse, fine)
    ts = [cpu_run(lib, kind, boxes, crse, fine) for _ in range(args.steps)]
    t = float(np.sum(ts))
    value = pts * args.steps / t
    cores = cpu_threads() if kind == "reference" else cpu_threads()
    sample = f"component 0 of all {len(boxes)} boxes ({pts} fine points) per step"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# GPU arm

def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    import torch
    import carpetx_b200 as cb

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    # weak scaling: one level of `boxes` x N boxes, knapsack-distributed over
    # the N ranks (every rank computes the same mapping); a box's transfer is
    # local to its owner, so there is no data-path collective
    from carpetx_b200.distribute import box_cost, max_over_ranks as _max_over_ranks, my_boxes
    from carpetx_b200.distribute import sum_over_ranks
    all_boxes, cfg = workload(args.workload, args.seed, args.boxes * world, args.ncomp)
    costs = [box_cost(b[5], b[6], b[7]) for b in all_boxes]
    boxes = my_boxes(all_boxes, costs, rank, world)
    total_fine = sum(costs)  # regions are the whole fine boxes
    coff, foff, ctot, ftot = [], [], 0, 0
    for b in boxes:
        coff.append(ctot)
        foff.append(ftot)
        ctot += b[7] * npts(b[3], b[4])
        ftot += b[7] * npts(b[5], b[6])
    crse = torch.empty(ctot, dtype=torch.float64, device=dev)
    fine = torch.empty(ftot, dtype=torch.float64, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(args.seed + rank)
    crse.normal_(generator=gen)
    lb = []
    for b, co, fo in zip(boxes, coff, foff):
        typ, order, it, clo, chi, flo, fhi, n = b
        lb.append(dict(op=cb.Op(typ, order, it), ncomp=n,
                       crse=crse[co:co + n * npts(clo, chi)].view((n,) + box_shape(clo, chi)),
                       crse_lo=clo, crse_hi=chi,
                       fine=fine[fo:fo + n * npts(flo, fhi)].view((n,) + box_shape(flo, fhi)),
                       fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi))
    plan = cb.LevelPlan(lb)
    st = plan.stats()
    nfine = st["fine_points"]
    alg_bytes = st["bytes"]
    stream = torch.cuda.Stream(device=dev)

    # capture the level transfer as a CUDA graph
    with torch.cuda.stream(stream):
        plan.execute(stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        plan.execute(stream)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return _max_over_ranks(x, dev)

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    time.sleep(0.3)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with torch.cuda.stream(stream):
        ev[0].record(stream)
        for k in range(args.steps):
            graph.replay()
            ev[k + 1].record(stream)
    barrier()
    clk = clocks.stop()
    per_step = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    ms_total = max_over_ranks(ev[0].elapsed_time(ev[-1]))
    ms_step = ms_total / args.steps
    value = total_fine * args.steps / (ms_total / 1e3)

    # the same level under the untuned schedule (every instantiation
    # schedule 0 with a z-chunk cap of 128) against the tuned table that
    # plan above uses (csrc/stream_tuned.h, written by carpetx_b200/tune.py)
    tuning = None
    if args.tune_steps > 0:
        L0 = cb.lib()
        L0.cx_debug_set_stream_schedule(-1, 0, 128)
        plan_u = cb.LevelPlan(lb)
        L0.cx_debug_set_stream_schedule(-1, -1, 0)
        with torch.cuda.stream(stream):
            for _ in range(2):
                plan_u.execute(stream)
                plan.execute(stream)
        res_t = {}
        for name, pl in (("untuned", plan_u), ("tuned", plan)):
            barrier()
            e0t, e1t = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0t.record(stream)
                for _ in range(args.tune_steps):
                    pl.execute(stream)
                e1t.record(stream)
            barrier()
            res_t[name] = max_over_ranks(e0t.elapsed_time(e1t)) / args.tune_steps
        plan_u.close()
        tuning = {"workload": "the level of this line, eager plan executions",
                  "tuned_ms": res_t["tuned"], "untuned_ms": res_t["untuned"],
                  "speedup": res_t["untuned"] / res_t["tuned"],
                  "table": "carpetx_b200/csrc/stream_tuned.h"}

    # the same work launched once per box per component (our kernel)
    L = cb.lib()
    I3 = ctypes.c_int * 3
    calls = []
    for b in lb:
        n = b["ncomp"]
        cs = npts(b["crse_lo"], b["crse_hi"])
        fs = npts(b["fine_lo"], b["fine_hi"])
        for c in range(n):
            calls.append((b["op"].handle, ctypes.c_void_p(b["crse"].data_ptr() + 8 * c * cs),
                          I3(*b["crse_lo"]), I3(*b["crse_hi"]),
                          ctypes.c_void_p(b["fine"].data_ptr() + 8 * c * fs),
                          I3(*b["fine_lo"]), I3(*b["fine_hi"]), I3(*b["reg_lo"]),
                          I3(*b["reg_hi"])))
    sp = ctypes.c_void_p(stream.cuda_stream)

    def per_box_step():
        for c in calls:
            rc = L.cx_prolong_box(*c, 1, 0, sp)
            if rc:
                raise RuntimeError(L.cx_last_error().decode())

    # the per-box launches are captured once as a CUDA graph and replayed,
    # so the figure is the device-side cost of the reference's launch
    # granularity, without this script's per-call host overhead
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms_pb, per_box_value = None, None
    if args.per_box_steps > 0:
        with torch.cuda.stream(stream):
            per_box_step()
        torch.cuda.synchronize()
        g_pb = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g_pb, stream=stream):
            per_box_step()
        g_pb.replay()
        torch.cuda.synchronize()
        barrier()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.per_box_steps):
                g_pb.replay()
            e1.record(stream)
        barrier()
        ms_pb = max_over_ranks(e0.elapsed_time(e1)) / args.per_box_steps
        per_box_value = total_fine / (ms_pb / 1e3)
        del g_pb

    # end to end through the C ABI with host buffers: every step copies all
    # coarse data in from pinned host memory and all fine data out.  The
    # level is split into --e2e-batches batches of consecutive boxes, one plan
    # each, pipelined over three streams: batch k's copy in, transfer and
    # copy out wait for each other, and the copy in (copy out) of a batch
    # waits for the previous step's transfer (copy out) of that batch, whose
    # buffers it overwrites.  Copies in and out then run at the same time on
    # the two copy directions, beside the transfers.  Each batch's copies are
    # issued in pieces of at most --e2e-chunk-mb.
    ms_e2e, e2e_value = None, None
    if args.e2e_steps > 0:
        h_crse = torch.empty(ctot, dtype=torch.float64, pin_memory=True)
        h_fine = torch.empty(ftot, dtype=torch.float64, pin_memory=True)
        h_crse.copy_(crse.cpu())
        nb = len(lb)
        nbat = max(1, args.e2e_batches)
        cuts = sorted({round(i * nb / nbat) for i in range(nbat + 1)})
        chunk = args.e2e_chunk_mb * (1 << 20) // 8 if args.e2e_chunk_mb > 0 else None

        def copy_chunks(dst, src, a, z):
            step = chunk or (z - a)
            for u in range(a, z, step):
                dst[u:min(u + step, z)].copy_(src[u:min(u + step, z)], non_blocking=True)
        coff_all, foff_all = coff + [ctot], foff + [ftot]
        batches = [(cb.LevelPlan(lb[a:z]), coff_all[a], coff_all[z], foff_all[a], foff_all[z])
                   for a, z in zip(cuts[:-1], cuts[1:]) if z > a]
        s_in, s_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        done_x = [None] * len(batches)  # previous step's transfer of batch k
        done_o = [None] * len(batches)  # previous step's copy out of batch k

        def e2e_step():
            for k, (bp, c0, c1, f0, f1) in enumerate(batches):
                ev_in, ev_x, ev_o = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
                with torch.cuda.stream(s_in):
                    if done_x[k] is not None:
                        s_in.wait_event(done_x[k])
                    copy_chunks(crse, h_crse, c0, c1)
                    ev_in.record(s_in)
                stream.wait_event(ev_in)
                if done_o[k] is not None:
                    stream.wait_event(done_o[k])
                bp.execute(stream)
                ev_x.record(stream)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(ev_x)
                    copy_chunks(h_fine, fine, f0, f1)
                    ev_o.record(s_out)
                done_x[k], done_o[k] = ev_x, ev_o

        e2e_step()
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        s_in.wait_stream(stream)
        for _ in range(args.e2e_steps):
            e2e_step()
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        e1.record(stream)
        barrier()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1)) / args.e2e_steps
        e2e_value = total_fine / (ms_e2e / 1e3)
        for bp, *_ in batches:
            bp.close()

    adjoint = adjoint_leg(args, cb, torch, dev, max_over_ranks, barrier) if args.adjoint_steps > 0 \
        else None
    peak, peak_src = measured_peaks()
    restriction = (restrict_leg(args, cb, torch, dev, max_over_ranks, barrier, peak)
                   if args.restrict_steps > 0 else None)
    limited = (limited_leg(args, cb, torch, dev, max_over_ranks, barrier)
               if args.limited_steps > 0 else None)
    boundary = (boundary_leg(args, cb, torch, dev, max_over_ranks, barrier, peak)
                if args.boundary_steps > 0 else None)
    halo = (halo_leg(args, cb, torch, dev, max_over_ranks, barrier, peak)
            if args.halo_steps > 0 else None)
    sync = None
    if args.sync_steps > 0:
        try:
            sync = sync_leg(args, cb, torch, dev, max_over_ranks, barrier, peak)
        except Exception as e:  # a failing extra leg does not void the headline line
            sync = {"error": f"{type(e).__name__}: {e}"}

    # per GPU: the ranks' mean algorithmic bytes over the slowest rank's time
    mean_bytes = sum_over_ranks(alg_bytes, dev) / world
    achieved = mean_bytes / (ms_step / 1e3) / 1e9
    # DRAM traffic grows with the fine points: the measured bytes per point
    # scaled to this step
    traffic = (TRAFFIC_PER_FINE_POINT * nfine if args.workload == "level512" else None)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(cfg, fine_points_per_gpu=nfine, algorithmic_bytes_per_gpu=alg_bytes,
                       l2_flush=f"inputs+outputs {(8 * (ctot + ftot)) / 1e9:.1f} GB per GPU "
                                f">> L2 ({L2_BYTES / 2**20:.0f} MiB); no explicit flush",
                       boxes_total=len(all_boxes), boxes_this_rank=len(boxes),
                       parallelism=f"weak: one level of {len(all_boxes)} boxes, knapsack-"
                                   f"distributed over {world} rank(s), no data-path collective",
                       launch=f"{st['launches']} persistent launches per step (one per kernel "
                              "instantiation and CTA size present), each after the first a "
                              "programmatic dependent launch; CUDA graph replay"),
        "gpu_launches": args.steps * st["launches"],
        "per_box": {"value": per_box_value, "unit": UNIT, "ms_per_step": ms_pb,
                    "launches_per_step": len(calls),
                    "timing": "one CUDA graph of the per-box launches, replayed",
                    "batched_speedup": value / per_box_value if per_box_value else None},
        "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": 8 * ctot, "d2h_bytes_per_step": 8 * ftot,
                "batches": args.e2e_batches, "copy_chunk_mb": args.e2e_chunk_mb},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_unit": "bytes per step (rank 0)",
                     "peak_source": peak_src,
                     "frac_of_8TBs_spec": achieved / 8000.0,
                     "step_ms_min": min(per_step), "step_ms_max": max(per_step)},
        "clocks": clk,
        "adjoint": adjoint,
        "restriction": restriction,
        "limited": limited,
        "tuning": tuning,
        "boundary": boundary,
        "halo": halo,
        "sync": sync,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        lib, kind = cpu_lib()
        cboxes = boxes
        c_crse, c_fine = cpu_sample(cboxes, args.seed)
        t, npass = cpu_timed_passes(lib, kind, cboxes, c_crse, c_fine)
        pts = sum(npts(b[5], b[6]) for b in cboxes)
        line["cpu_baseline"] = {"value": pts * npass / t, "unit": UNIT, "cores": cpu_threads(),
                                "cpu_model": cpu_model(), "kind": kind,
                                "sample": f"component 0 of all {len(cboxes)} boxes "
                                          f"({pts} fine points) per pass, {npass} passes "
                                          f"({t:.1f} s) after two warm-up passes"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    del graph
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
