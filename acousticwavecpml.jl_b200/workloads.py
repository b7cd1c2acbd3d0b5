"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Grid conventions: a CPML axis has interior + 2*halo nodes; the depth axis
(j, the reference's second axis) with a free top has interior + halo nodes,
node j = 1 being the Dirichlet surface. Positions are given in metres as
(node - 1) * d, so they snap back exactly to the intended 1-based node.
Each builder returns a dict with the solve2D/solve3D arguments:
lengths, lt, vel, srcs (positions, t0s, f0), recs (positions), kwargs.
"""
import math

import numpy as np


def gaussian_smooth(a, sigma):
    """Gaussian filter (reflecting edges, truncated at 3 sigma)."""
    from scipy.ndimage import gaussian_filter

    return gaussian_filter(a, sigma=sigma, mode="reflect", truncate=3.0)


def config1():
    """2D FP64, the reference's CPU-runnable size: 201^2 interior + CPML 20
    (241 x 241 nodes), dx = dy = 10 m, c = 2000 m/s, R = 1e-3, no free top,
    Ricker f0 = 8 Hz, t0 = 0.5 s at the centre node (121, 121),
    dt = 0.7 dx / (c sqrt 2), nt = 1000, 21 receivers on row j = 31 (10 nodes
    below the top of the interior), i = 21, 31, ..., 221."""
    n, dx, c = 241, 10.0, 2000.0
    L = (n - 1) * dx
    f0 = 8.0
    dt = 0.7 * dx / (c * math.sqrt(2.0))
    recs = [[(i - 1) * dx, 30 * dx] for i in range(21, 222, 10)]
    return dict(name="cpml2d_241x241_f64_nt1000", lengths=(L, L), lt=None,
                vel=np.full((n, n), c, order="F"), src_pos=[[120 * dx, 120 * dx]], t0s=[0.5],
                f0=f0, rec_pos=recs, kwargs=dict(halo=20, rcoef=1e-3, freetop=False, dt=dt,
                                                 nt=1000))


def config2_model(seed=1234, interior=256, halo=20, dx=10.0):
    """c(depth) = 1500 + 1.5 depth_m times (1 + 5% seeded Gaussian-smoothed
    noise, sigma = 8 nodes), on (interior + 2 halo, interior + halo,
    interior + 2 halo) nodes, depth on the second axis."""
    nx = nz = interior + 2 * halo
    ny = interior + halo
    base = 1500.0 + 1.5 * (np.arange(ny, dtype=np.float64) * dx)
    rng = np.random.default_rng(seed)
    noise = gaussian_smooth(rng.standard_normal((nx, ny, nz), dtype=np.float64), 8.0)
    noise *= 0.05 / np.abs(noise).max()
    return np.asfortranarray(base[None, :, None] * (1.0 + noise))


def config2(nt=2000, seed=1234, interior=256):
    """3D single shot, the headline benchmark: 256^3 interior (296 x 276 x 296
    nodes), dx = 10 m, model of config2_model, halo 20, free top, Ricker
    f0 = 10 Hz at interior (128, 128, 10) = node (148, 11, 148),
    dt = 0.6 dx / (cmax sqrt 3), nt = 2000, 64 x 64 receivers on depth node
    j = 6 at i, k = 23, 27, ..., 275."""
    dx, halo = 10.0, 20
    vel = config2_model(seed=seed, interior=interior, halo=halo, dx=dx)
    nx, ny, nz = vel.shape
    f0 = 10.0
    dt = 0.6 * dx / (float(vel.max()) * math.sqrt(3.0))
    c = interior // 2
    src = [[(c + halo - 1) * dx, 10 * dx, (c + halo - 1) * dx]]
    idx = [i for i in (21 + 4 * a + 2 for a in range(64)) if i <= nx - 1]
    recs = [[(i - 1) * dx, 5 * dx, (k - 1) * dx] for k in idx for i in idx]
    L = ((nx - 1) * dx, (ny - 1) * dx, (nz - 1) * dx)
    return dict(name=f"cpml3d_{nx}x{ny}x{nz}_freetop_nt{nt}", lengths=L, lt=None, vel=vel,
                src_pos=src, t0s=[4 / f0], f0=f0, rec_pos=recs,
                kwargs=dict(halo=halo, rcoef=1e-4, freetop=True, dt=dt, nt=nt))


CONFIG3_INTERIORS = ((512, 256), (768, 384), (1024, 512), (1536, 768), (2048, 1024),
                     (1024, 1024))


def layered_model(rng, nx, ny, halo, dx):
    """Layered velocity 1500-4500 m/s with 3-8 interfaces at seeded depths,
    increasing downwards with seeded jumps, times (1 + 3% seeded
    Gaussian-smoothed noise, sigma = 4 nodes)."""
    nint = int(rng.integers(3, 9))
    depths = np.sort(rng.choice(np.arange(8, ny - 8), size=nint, replace=False))
    v = np.sort(rng.uniform(1500.0, 4500.0, size=nint + 1))
    v[0], v[-1] = 1500.0, 4500.0
    col = np.full(ny, v[0])
    for k, j in enumerate(depths):
        col[j:] = v[k + 1]
    noise = gaussian_smooth(rng.standard_normal((nx, ny)), 4.0)
    noise *= 0.03 / np.abs(noise).max()
    return np.asfortranarray(col[None, :] * (1.0 + noise))


def config3(nt=3000, seed=4321, shots_per_model=16, interiors=CONFIG3_INTERIORS, halo=20,
            dx=5.0):
    """2D batched shots: one layered model per interior size (nx x ny interior,
    512 x 256, 768 x 384, 1024 x 512, 1536 x 768, 2048 x 1024, 1024 x 1024;
    grid interior + 2 halo by interior + halo with a free top), dx = dy = 5 m, halo 20, R = 1e-4, each model's own CFL step
    dt = sqrt(2) / (cmax (1/dx + 1/dy)) / 2, nt common. Each model carries
    `shots_per_model` Ricker shots evenly spaced along depth node j = 3 with
    f0 ~ U(10, 20) Hz and t0 = 1.2 / f0, and receivers on every 4th node of
    j = 3 inside the interior."""
    rng = np.random.default_rng(seed)
    models, shots = [], []
    for m, (ix, iy) in enumerate(interiors):
        nx, ny = ix + 2 * halo, iy + halo
        vel = layered_model(rng, nx, ny, halo, dx)
        models.append(((nx - 1) * dx, (ny - 1) * dx, vel))
        rec = [[(i - 1) * dx, 2 * dx] for i in range(halo + 1, nx - halo + 1, 4)]
        for s in range(shots_per_model):
            i = halo + 1 + round((s + 0.5) * (ix - 1) / shots_per_model)
            f0 = float(rng.uniform(10.0, 20.0))
            shots.append(dict(model=m, src_pos=[[(i - 1) * dx, 2 * dx]], t0s=[1.2 / f0],
                              f0=f0, rec_pos=rec))
    return dict(name=f"cpml2d_batch_{len(models)}models_{len(shots)}shots_nt{nt}",
                models=models, shots=shots,
                kwargs=dict(halo=halo, rcoef=1e-4, freetop=True, nt=nt))


def config4(nt=1500, seed=77, interior=(192, 192, 192), halo=20, dx=10.0):
    """3D gradient workload: 192^3 interior (232 x 212 x 232 nodes, depth on
    the second axis, free top), dx = 10 m, c = 2000 + depth_m for the initial
    model; the true model adds a blob of +10 % at its centre, (1 - r²/R²)²
    with R = 20 nodes and zero beyond (seeded centre in the interior). 16 Ricker shots (f0 = 8 Hz, t0 = 1.2 / f0)
    on a 4 x 4 grid at depth node j = 3, 48 x 48 receivers at j = 3 over the
    interior, nt common, dt = 0.6 dx / (cmax sqrt 3) of the true model,
    checkpoint every 50 steps."""
    ix, iy, iz = interior
    nx, ny, nz = ix + 2 * halo, iy + halo, iz + 2 * halo
    depth = np.arange(ny, dtype=np.float64) * dx
    init = np.asfortranarray(np.broadcast_to((2000.0 + depth)[None, :, None], (nx, ny, nz)))
    rng = np.random.default_rng(seed)
    cx, cy, cz = (int(rng.integers(halo + min(40, n // 4), halo + n - min(40, n // 4)))
                  for n in (ix, iy, iz))
    cy -= halo  # depth axis has no top band
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    r2 = ((X - cx) ** 2 + (Y - cy) ** 2 + (Z - cz) ** 2) / 20.0 ** 2
    blob = np.where(r2 < 1.0, (1.0 - r2) ** 2, 0.0)  # smooth, zero beyond 20 nodes
    true = np.asfortranarray(init * (1.0 + 0.10 * blob))
    dt = 0.6 * dx / (float(true.max()) * math.sqrt(3.0))
    f0 = 8.0
    xs = [halo + 1 + round((a + 0.5) * (ix - 1) / 4) for a in range(4)]
    shots = [[[(i - 1) * dx, 2 * dx, (k - 1) * dx]] for k in xs for i in xs]
    ridx = [halo + 1 + round(a * (ix - 1) / 47) for a in range(48)]
    recs = [[(i - 1) * dx, 2 * dx, (k - 1) * dx] for k in ridx for i in ridx]
    L = ((nx - 1) * dx, (ny - 1) * dx, (nz - 1) * dx)
    return dict(name=f"cpml3d_grad_{nx}x{ny}x{nz}_16shots_nt{nt}", lengths=L, true=true,
                init=init, shots=shots, t0s=[1.2 / f0], f0=f0, rec_pos=recs,
                kwargs=dict(halo=halo, rcoef=1e-4, freetop=True, dt=dt, nt=nt),
                checkpoint_every=50)


def batch_shots(pkg, w):
    """(model index, Sources, Receivers) per shot of a batched workload."""
    out = []
    for sh in w["shots"]:
        srcs = pkg.Sources(sh["src_pos"], sh["t0s"], [pkg.rickersource1D], sh["f0"])
        out.append((sh["model"], srcs, pkg.Receivers(sh["rec_pos"])))
    return out


def sources_receivers(pkg, w):
    """Sources/Receivers objects (Ricker source functions) of a workload."""
    srcs = pkg.Sources(w["src_pos"], w["t0s"], [pkg.rickersource1D] * len(w["t0s"]), w["f0"])
    recs = pkg.Receivers(w["rec_pos"])
    return srcs, recs
