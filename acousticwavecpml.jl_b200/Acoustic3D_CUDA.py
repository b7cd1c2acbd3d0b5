"""`Acoustic3D_CUDA.solve3D` (src/Acoustic3D_CUDA.jl, body
src/shared/acoustic_3D_xPU.jl:169-545) over the B200 library."""
from ._solver import solve

__all__ = ["solve3D"]


def solve3D(lx, ly, lz, lt, vel, srcs, recs, *, halo=20, rcoef=0.0001, ppw=10.0, freetop=True,
            do_bench=False, do_vis=False, do_save=False, nvis=5, nsave=5,
            gif_name="acoustic3D_xPU_slice", save_name="acoustic3D_xPU", plims=(-1.0, 1.0),
            threshold=0.01, precision="f64", dt=None, nt=None, device=0, verbose=True):
    """Solve the 3D acoustic wave equation on an lx x ly x lz [m] model for lt [s].

    Same arguments and behaviour as the reference (depth is the second axis;
    ``freetop`` removes the CPML on j = 1): returns the final pressure field
    and fills ``recs.seismograms`` (nt x nrec). Extensions as in solve2D.
    ``do_vis`` (graphics) and ``do_save`` (HDF5 snapshots) are not available.
    """
    if do_save:
        raise NotImplementedError("do_save (HDF5 snapshots) is not available in this build")
    return solve((lx, ly, lz), lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw,
                 freetop=freetop, do_bench=do_bench, do_vis=do_vis, precision=precision,
                 dt=dt, nt=nt, device=device, verbose=verbose)
