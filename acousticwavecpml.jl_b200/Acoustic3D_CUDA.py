"""`Acoustic3D_CUDA.solve3D` (src/Acoustic3D_CUDA.jl, body
src/shared/acoustic_3D_xPU.jl:169-545) over the B200 library."""
from ._solver import solve

__all__ = ["solve3D"]


def solve3D(lx, ly, lz, lt, vel, srcs, recs, *, halo=20, rcoef=0.0001, ppw=10.0, freetop=True,
            do_bench=False, do_vis=False, do_save=False, nvis=5, nsave=5,
            gif_name="acoustic3D_xPU_slice", save_name="acoustic3D_xPU", plims=(-1.0, 1.0),
            threshold=0.01, precision="f64", dt=None, nt=None, device=0, verbose=True,
            save_dir=None):
    """Solve the 3D acoustic wave equation on an lx x ly x lz [m] model for lt [s].

    Same arguments and behaviour as the reference (depth is the second axis;
    ``freetop`` removes the CPML on j = 1): returns the final pressure field
    and fills ``recs.seismograms`` (nt x nrec). Extensions as in solve2D.
    ``do_save`` writes the pressure after every step it with it % nsave == 0
    to ``save_dir/{save_name}_it{it}`` (HDF5 with the reference's datasets
    lx, ly, lz, halo, pcur, possrcs, posrecs when h5py is installed, else
    .npz with the same names; save_dir defaults to simulations/tmp under the
    working directory). ``do_vis`` (graphics) is not available.
    """
    kw = {}
    if save_dir is not None:
        kw["save_dir"] = save_dir
    return solve((lx, ly, lz), lt, vel, srcs, recs, halo=halo, rcoef=rcoef, ppw=ppw,
                 freetop=freetop, do_bench=do_bench, do_vis=do_vis, precision=precision,
                 dt=dt, nt=nt, device=device, verbose=verbose, do_save=do_save, nsave=nsave,
                 save_name=save_name, **kw)
