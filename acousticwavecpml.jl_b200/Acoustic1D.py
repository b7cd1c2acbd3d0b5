"""`Acoustic1D.solve1D` (src/Acoustic1D.jl, body src/shared/acoustic_1D.jl:89-297)
over the B200 library: the 1D CPML time loop runs on the GPU as the line of a
three-row 2D problem (awc_forward with ndim = 1)."""
from ._solver import solve

__all__ = ["solve1D"]


def solve1D(lx, lt, vel, srcs, recs, *, halo=20, rcoef=0.0001, ppw=10.0, do_bench=False,
            do_vis=False, nvis=5, gif_name="acoustic1D", plims=(-1.0, 1.0), precision="f64",
            dt=None, nt=None, device=0, verbose=True):
    """Solve the 1D acoustic wave equation on a line of length lx [m] for lt [s].

    Same arguments and behaviour as the reference: dt = dx / max(vel) / 2,
    nt = ceil(lt / dt), CPML of `halo` nodes at both ends, returns the final
    pressure (the reference's `pcur`) and fills ``recs.seismograms``
    (nt x nrec). Positions are (n x 1) in metres. Extensions as in solve2D;
    ``do_vis`` needs a graphics stack and is not available.
    """
    return solve((lx,), lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw, freetop=False,
                 do_bench=do_bench, do_vis=do_vis, precision=precision, dt=dt, nt=nt,
                 device=device, verbose=verbose)
