"""Path-replay adjoint against central finite differences on the 2-D bench
model (nr=100, ntheta=99, diffusion on) at 4e7 packets per evaluation, the
scale at which its Monte Carlo error is below the 2 % target.

Scaling one density component everywhere by exp(+-eps) changes the objective
(the peeled SED plus the 3.6/24/70 um images) by 2 eps * sum(grad[:, comp]).
Both sides use the same seeds (common random numbers), so the test is
deterministic up to the order of FP64 atomic sums.  The envelope and cavity
components are checked.  The optically thick disk is not: its estimate
scatters by ~6 % from seed to seed on both sides at this size.
"""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import adjoint as madj
from src3_mpi_cfitsio_b200 import model

pytestmark = pytest.mark.gpu


def test_adjoint_within_two_percent_of_central_differences():
    from src3_mpi_cfitsio_b200.engine import Engine
    base = model.with_diffusion(model.warm(model.reference_2d()))
    lam, img = madj.sed_image_weights(base)
    c = base.config
    ncell = c["nrg"] * c["ntg"] * c["npg"]
    dens0 = base.grid["densarr"].reshape((ncell, 10), order="F").copy()
    n, eps, seeds = 40_000_000, 0.05, (12345678, 87654321)
    eng = Engine(base, precision="mixed")
    g, L = eng.adjoint(n, lam, img, seeds=seeds)
    G = g.reshape((ncell, 10), order="F")
    assert L > 0
    for comp in (2, 3):                       # 0-based columns: envelope (id 3) and cavity (id 4)
        vals = []
        for sgn in (1, -1):
            d = dens0.copy()
            d[:, comp] *= np.exp(sgn * eps)
            base.grid["densarr"] = d.ravel(order="F")
            eng.upload_grid()
            vals.append(eng.adjoint(n, lam, img, seeds=seeds)[1])
        fd = (vals[0] - vals[1]) / (2 * eps)
        adj = G[:, comp].sum()
        assert abs(adj - fd) <= 0.02 * abs(fd), (comp + 1, adj, fd)
    eng.close()
