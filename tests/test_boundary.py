"""CPU tests of the outer boundary conditions' oracle (cxo_boundary_box, the C
restatement of CarpetX's BoundaryCondition, CarpetX/src/boundaries*.cxx):
against the golden fixture made by the reference itself, against the
reference build when present, known answers of each condition, and the
argument checks."""
import os

import numpy as np
import pytest

from boundary_cases import fab_data, outside_mask, random_bc_case
from helpers import assert_bitwise

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "boundary_golden.npz")


def golden_cases():
    z = np.load(GOLDEN)
    for key in sorted(z.files):
        seed = int(key[:4])
        spec, lo, hi = random_bc_case(seed, max_n=6, max_ghost=2, max_comp=2)
        yield seed, spec, lo, hi, z[key]


def test_boundary_golden_covers_every_condition():
    seen = set()
    for _, spec, _, _, _ in golden_cases():
        for f in range(2):
            for d in range(3):
                seen.add((spec["symmetry"][f][d], spec["boundary"][f][d]))
    # every (symmetry, boundary) pair CarpetX accepts, periodic included
    from carpetx_b200.workloads import BC_FACE_CHOICES
    assert set(BC_FACE_CHOICES) | {(2, 0)} <= seen


def test_boundary_oracle_matches_golden(cx):
    n = 0
    for seed, spec, lo, hi, want in golden_cases():
        a = fab_data(seed, len(spec["dirichlet"]), lo, hi)
        before = a.copy()
        cx.boundary(spec, a, lo, hi)
        m = outside_mask(spec, lo, hi)
        assert_bitwise(a[:, m], want, f"case {seed}")
        assert_bitwise(a[:, ~m], before[:, ~m], f"case {seed} interior")
        n += 1
    assert n == 64


def test_boundary_oracle_matches_reference(cx):
    from oracle.oracle import RefBoundary
    if not RefBoundary.available():
        pytest.skip("reference oracle (oracle/_ref) not built")
    ref = RefBoundary()
    for seed in range(1000, 1300):
        spec, lo, hi = random_bc_case(seed, max_n=9, max_ghost=3, max_comp=4)
        a = fab_data(seed, len(spec["dirichlet"]), lo, hi)
        b = a.copy()
        cx.boundary(spec, a, lo, hi)
        ref.boundary(spec, b, lo, hi)
        assert_bitwise(a, b, f"case {seed}")


def _spec(faces, it=(1, 1, 1), n=(6, 6, 6), ncomp=1, **kw):
    from carpetx_b200.workloads import boundary_spec
    s = boundary_spec(np.random.default_rng(0), ncomp, it, n, nghost=2, faces=faces)
    s.update(kw)
    return s


NONE6 = [[(0, 0)] * 3, [(0, 0)] * 3]


def test_boundary_known_answers(cx):
    lo, hi = (-2, -2, -2), (7, 7, 7)
    base = fab_data(5, 1, lo, hi)
    at = lambda a, i, j, k: a[0, k + 2, j + 2, i + 2]  # noqa: E731
    # Dirichlet on x lower: the value, on every ghost point of that face
    f = [row[:] for row in NONE6]
    f[0][0] = (0, 2)
    a = base.copy()
    cx.boundary(_spec(f, dirichlet=[3.25]), a, lo, hi)
    assert at(a, -1, 3, 3) == 3.25 and at(a, -2, 0, 5) == 3.25
    assert at(a, 0, 3, 3) == at(base, 0, 3, 3)
    # Neumann on y upper: the value of the last interior point (cells: y = 5)
    f = [row[:] for row in NONE6]
    f[1][1] = (0, 4)
    a = base.copy()
    cx.boundary(_spec(f), a, lo, hi)
    assert at(a, 2, 6, 1) == at(base, 2, 5, 1) and at(a, 2, 7, 1) == at(base, 2, 5, 1)
    # reflection, cell centred, odd parity: x = -1 - i mirrors i
    f = [row[:] for row in NONE6]
    f[0][0] = (3, 0)
    a = base.copy()
    cx.boundary(_spec(f, parity=[[-1, 1, 1]]), a, lo, hi)
    assert at(a, -1, 2, 2) == -at(base, 0, 2, 2) and at(a, -2, 2, 2) == -at(base, 1, 2, 2)
    # reflection, vertex centred, even parity: x = -i mirrors i
    a = base.copy()
    cx.boundary(_spec(f, it=(0, 1, 1), parity=[[1, 1, 1]]), a, lo, hi)
    assert at(a, -1, 2, 2) == at(base, 1, 2, 2) and at(a, -2, 2, 2) == at(base, 2, 2, 2)
    # linear extrapolation on z lower: f(-k) = f(0) + k (f(0) - f(1))
    f = [row[:] for row in NONE6]
    f[0][2] = (0, 3)
    a = base.copy()
    cx.boundary(_spec(f), a, lo, hi)
    f0, f1 = at(base, 3, 3, 0), at(base, 3, 3, 1)
    assert at(a, 3, 3, -1) == f0 + 1.0 * (f0 - f1)
    assert at(a, 3, 3, -2) == f0 + 2.0 * (f0 - f1)
    # periodic everywhere: nothing is written
    a = base.copy()
    cx.boundary(_spec([[(2, 0)] * 3, [(2, 0)] * 3]), a, lo, hi)
    assert_bitwise(a, base, "all periodic")


def test_boundary_oracle_rejects(cx):
    lo, hi = (-2, -2, -2), (7, 7, 7)
    a = fab_data(1, 1, lo, hi)
    before = a.copy()
    f = [row[:] for row in NONE6]
    f[0][1] = (0, 1)  # symmetry_boundary without a reflection symmetry
    with pytest.raises(ValueError):
        cx.boundary(_spec(f), a, lo, hi)
    f = [row[:] for row in NONE6]
    f[0][0] = (3, 0)
    with pytest.raises(ValueError):  # parity 0
        cx.boundary(_spec(f, parity=[[0, 1, 1]]), a, lo, hi)
    with pytest.raises(ValueError):  # domain of 1 cell: mirror of x = -2 is outside
        cx.boundary(_spec(f, n=(1, 6, 6), domain_hi=(0, 5, 5)), a, lo, hi)
    assert_bitwise(a, before, "rejected calls write nothing")


def test_boundary_host_checks_accept_test_cases():
    """The C ABI's region builder accepts every case the GPU tests run: each
    region's accesses, checked at its corners with the kernel's own index
    code, stay inside the FAB.  Runs plan creation only (never a launch), with
    a placeholder data pointer: CX_OK on a machine with a device, CX_ECUDA or
    CX_ENOMEM (the region list upload) without one, never CX_EINVAL."""
    import ctypes
    import carpetx_b200 as cb
    from carpetx_b200.workloads import BC_LEVEL_FACES, boundary_spec, tiled_level_fabs
    L = cb.lib()

    def check(spec, fabs):
        b = cb.bc_struct(spec)
        arr = (cb.CxBcFab * len(fabs))()
        for i, (lo, hi) in enumerate(fabs):
            arr[i] = cb.CxBcFab(0x10000, cb._i3(lo), cb._i3(hi))
        h = ctypes.c_void_p()
        st = L.cx_boundary_plan_create(ctypes.byref(b), arr, len(fabs), ctypes.byref(h))
        assert st in (cb.CX_OK, cb.CX_ECUDA, cb.CX_ENOMEM), L.cx_last_error().decode()
        if st == cb.CX_OK:
            L.cx_boundary_plan_destroy(h)

    for seed in range(2000, 2150):
        spec, lo, hi = random_bc_case(seed, max_n=10, max_ghost=3, max_comp=5)
        check(spec, [(lo, hi)])
    for seed in range(6):
        rng = np.random.default_rng(300 + seed)
        it = tuple(int(v) for v in rng.integers(0, 2, 3))
        spec = boundary_spec(rng, int(rng.integers(1, 17)), it, (24, 16, 20), nghost=3,
                             periodic=(seed == 3, False, seed == 5))
        check(spec, tiled_level_fabs((24, 16, 20), (8, 8, 4), it, 3))
    spec = boundary_spec(np.random.default_rng(7), 16, (1, 1, 1), (256,) * 3, nghost=3,
                         faces=BC_LEVEL_FACES)
    check(spec, tiled_level_fabs((256,) * 3, (32,) * 3, (1, 1, 1), 3))
