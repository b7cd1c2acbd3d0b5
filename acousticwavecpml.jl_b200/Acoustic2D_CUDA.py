"""`Acoustic2D_CUDA.solve2D` (src/Acoustic2D_CUDA.jl, body
src/shared/acoustic_2D_xPU.jl:133-445) over the B200 library."""
from ._solver import solve

__all__ = ["solve2D"]


def solve2D(lx, ly, lt, vel, srcs, recs, *, halo=20, rcoef=0.0001, ppw=10.0, freetop=True,
            do_bench=False, do_vis=False, nvis=5, gif_name="acoustic2D_xPU", plims=(-1, 1),
            threshold=0.01, precision="f64", dt=None, nt=None, device=0, verbose=True):
    """Solve the 2D acoustic wave equation on an lx x ly [m] model for lt [s].

    Same arguments and behaviour as the reference: returns the final pressure
    field (the array `pcur` after the last step) and fills
    ``recs.seismograms`` (nt x nrec). Extensions: ``precision`` ("f64", the
    reference's Float64, or "f32"), an explicit ``dt``/``nt`` in place of the
    CFL-derived ones, and the CUDA ``device``. ``do_vis`` needs a graphics
    stack and is not available.
    """
    return solve((lx, ly), lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw,
                 freetop=freetop, do_bench=do_bench, do_vis=do_vis, precision=precision,
                 dt=dt, nt=nt, device=device, verbose=verbose)
