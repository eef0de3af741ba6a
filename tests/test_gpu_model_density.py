"""GPU density grid (mcrt_model_density) against the host generator of the
same density law (model.Model: disk, Ulrich envelope, polynomial cavity,
disk ownership, cell volumes) and the disk law's analytic log-derivatives
against central differences of the host law.

The two sides evaluate the same formulas in FP64.  pow/exp/acos may differ in
the last place between the CUDA and host libraries.  Measured on these grids
(B200): disk densities agree to 1.4e-14 relative and envelope densities to
3.3e-12, the latter through the Ulrich cubic near the equator.  Cell volumes
agree to 6e-12 on the bench grid, but the r^3 differences of the thinnest
rim shells cancel by up to 1e8, so volumes are held to the rounding bound of
the two cubes.  Densities are held to 1e-10.  A cell sitting exactly on the ownership or
cavity boundary could flip; none does.
"""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import model

pytestmark = pytest.mark.gpu


def _check(m):
    from src3_mpi_cfitsio_b200.engine import model_density
    dens, vcell, dlog = model_density(m)
    ref = m.grid["densarr"]
    assert ((dens > 0) != (ref > 0)).sum() <= 2        # a boundary cell within the last place may flip
    nz = (ref > 0) & (dens > 0)
    assert np.allclose(dens[nz], ref[nz], rtol=1e-10, atol=0)
    # vcell = (r1^3 - r0^3) (cos t0 - cos t1) dphi / 3 R*^3 (the reference's
    # form): the cancellation in r1^3 - r0^3 amplifies last-place differences
    # by r^3 / (r1^3 - r0^3), up to 1e8 for the thin rim shells, so the bound
    # is the rounding of the two cubes
    w = m.w
    r = m.grid["rarr"]
    dc = np.abs(np.cos(m.grid["thetarr"][1:]) - np.cos(m.grid["thetarr"][:-1]))
    scale = np.zeros((w.nrg, w.ntg, w.npg))
    scale[:-1, :-1, :-1] = ((r[1:] ** 3 + r[:-1] ** 3)[:, None] * dc[None, :])[:, :, None] * (
        2.0 * np.pi / (w.npg - 1)) / 3.0 * (w.rstar * 6.9598e10) ** 3
    scale = scale.ravel(order="F")
    assert np.all(np.abs(vcell - m.grid["vcell"]) <= 1e-14 * scale + 1e-13 * np.abs(m.grid["vcell"]))
    d = model.disk_log_derivatives(m)
    w = m.w
    shape = (w.nrg - 1, w.ntg - 1)
    for k, name in enumerate(model.DISK_PARAMS):
        g = dlog.reshape((*shape, 3), order="F")[:, :, k]
        h = d[name]
        on = h != 0
        # the host differences drop cells whose perturbed density underflows
        # the 1e-300 floor; the analytic derivative keeps them
        assert ((g != 0) != on).sum() <= max(5, 1e-3 * on.sum()), name
        both = on & (g != 0)
        assert np.allclose(g[both], h[both], rtol=1e-5, atol=1e-7 * np.abs(h).max()), name


@pytest.mark.parametrize("build", [lambda: model.reference_2d(), lambda: model.small_2d(npg=7),
                                   lambda: model.clumpy_3d(nrg=41, ntg=31, npg=9, nxhst=21, npeel=2)])
def test_density_grid_matches_the_host_generator(build):
    _check(build())


def test_density_grid_of_sweep_models():
    for m in model.batch_models(6, seed=7):
        _check(m)
