"""The amrex::Interpolater shim: compiled against AMReX/Cactus stand-in headers
and driven through CarpetX's registration tables and the virtual interface
(CarpetX/src/prolongate_3d_rf2.hxx:76-177), as fill-patch calls it."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from helpers import ALL_OPS, assert_bitwise, box_shape

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
I3 = ctypes.c_int * 3


@pytest.fixture(scope="session")
def shim(tmp_path_factory):
    import carpetx_b200
    carpetx_b200.lib()
    out = str(tmp_path_factory.mktemp("shim") / "libshim_harness.so")
    libdir = os.path.join(ROOT, "carpetx_b200")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-shared", "-fPIC",
           "-I", os.path.join(ROOT, "oracle", "ref_stubs"), "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "carpetx_b200", "host"),
           os.path.join(ROOT, "tests", "shim", "harness.cxx"),
           os.path.join(ROOT, "carpetx_b200", "host", "prolongate_3d_rf2_b200.cxx"),
           "-L", libdir, "-lcarpetx_b200", f"-Wl,-rpath,{libdir}", "-o", out,
           "-Wl,--no-as-needed", "-l:libstdc++.so.6"]
    subprocess.run(cmd, check=True)
    L = ctypes.CDLL(out)
    L.shim_coarse_box.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, I3, I3, I3, I3]
    L.shim_interp.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_void_p, I3, I3, ctypes.c_void_p, I3, I3, I3, I3,
                              ctypes.c_int, ctypes.c_int]
    return L


def test_shim_tables_coarse_box(shim, cx):
    for typ, order, it in ALL_OPS:
        for flo, fhi in [((0, 0, 0), (9, 9, 9)), ((-5, 3, -8), (2, 12, -1))]:
            clo, chi = I3(), I3()
            assert shim.shim_coarse_box(typ.encode(), order, it, I3(*flo), I3(*fhi), clo, chi) == 0
            assert (tuple(clo), tuple(chi)) == cx.coarse_box(typ, order, it, flo, fhi)
    assert shim.shim_coarse_box(b"interpolate", 2, 0, I3(), I3(), I3(), I3()) == -1


@pytest.mark.gpu
def test_shim_interp_on_device(shim, cx, dev):
    import torch
    rng = np.random.default_rng(17)
    for typ, order, it in [("interpolate", 3, 0), ("natural", 5, 5), ("eno", 3, 7),
                           ("poly-cons3lfb", 5, 3), ("conservative", 1, 7), ("minmod", 1, 6)]:
        for pg in (0, 1):
            for face in (0, 1):
                flo, fhi = (-3, 2, 0), (20, 17, 26)
                rlo, rhi = (-2, 2, 1), (19, 16, 26)
                clo, chi = cx.coarse_box(typ, order, it, rlo, rhi)
                crse = rng.standard_normal((3,) + box_shape(clo, chi))
                want = np.full((3,) + box_shape(flo, fhi), np.nan)
                cx.prolong(typ, order, it, pg, crse, clo, chi, want, flo, fhi, rlo, rhi, 3)
                g_crse = torch.from_numpy(crse).cuda()
                g_fine = torch.full(want.shape, np.nan, dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                assert shim.shim_interp(typ.encode(), order, it, pg, g_crse.data_ptr(), I3(*clo),
                                        I3(*chi), g_fine.data_ptr(), I3(*flo), I3(*fhi),
                                        I3(*rlo), I3(*rhi), 3, face) == 0
                torch.cuda.synchronize()
                assert_bitwise(g_fine.cpu().numpy(), want, f"shim {typ} {order} {it} pg{pg}")
