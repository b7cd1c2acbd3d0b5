"""Problem set-ups shared by the tests: the reference's own test cases
(test/test2D_xPU.jl, test/test3D_xPU.jl, test/test2D.jl, test/test3D.jl) and
small edge cases. Each returns (lengths, lt, vel, src_positions, t0s, f0,
rec_positions, kwargs)."""
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))["pend"]


def isapprox(a, b):
    """Julia's default isapprox for arrays: ‖a-b‖ <= sqrt(eps) max(‖a‖, ‖b‖)."""
    return np.linalg.norm(a - b) <= math.sqrt(np.finfo(np.float64).eps) * max(
        np.linalg.norm(a), np.linalg.norm(b))


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def ref_center(freetop):
    """test/test2D_xPU.jl:108-156 (golden acoustic2D_center[_freetop]_halo20)."""
    n, L = 201, 2000.0
    vel = 2000.0 * np.ones((n, n))
    f0 = 10.0
    return ((L, L), 2.0, vel, [[L / 2, L / 2]], [4 / f0], f0,
            [[L / 2, 2 * L / 3], [2 * L / 3, 2 * L / 3]], dict(halo=20, rcoef=1e-4, freetop=freetop))


def ref_gradient():
    """test/test2D_xPU.jl:158-195 (golden acoustic2D_gradient_freetop_halo20):
    6 surface sources at y = 5 m, which snap onto the Dirichlet row j = 1."""
    nx, ny = 211 * 2, 121 * 2
    vel = np.zeros((nx, ny))
    for j in range(ny):
        vel[:, j] = 2000.0 + 12.0 * j
    vel[:, ny - 41:] = vel[0, ny - 41]
    lx, ly = 2100.0 * 5, 1200.0 * 5
    f0 = 10.0
    srcs = [[k * lx / 11, 5.0] for k in range(3, 9)]
    return ((lx, ly), 5.0, vel, srcs, [4 / f0] * 6, f0,
            [[lx / 2, 2 * ly / 3], [2 * lx / 3, 2 * ly / 3]], dict(halo=20, rcoef=1e-4, freetop=True))
