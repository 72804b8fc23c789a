"""Single-box order-3 vertex-centred case: coarse vertices -1..33 (35^3, h = 1/32
on the unit cube, one ghost layer), fine region 0..63 (64^3 vertices), one
FP64 variable u = 0.3 + x - 2y^2 + 0.5xyz + z^3 + 0.01 sin(2 pi x) cos(2 pi y)
sin(2 pi z), evaluated on the host."""
import numpy as np


def config1_case():
    clo, chi = (-1, -1, -1), (33, 33, 33)
    h = 1.0 / 32
    x = np.arange(-1, 34) * h
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = (0.3 + X - 2 * Y ** 2 + 0.5 * X * Y * Z + Z ** 3
         + 0.01 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) * np.sin(2 * np.pi * Z))
    return dict(crse=u[None].copy(), clo=clo, chi=chi, flo=(0, 0, 0), fhi=(63, 63, 63))
