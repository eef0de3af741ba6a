"""mcrt_diskflux (the reference's diskflux, flux_test.f90) on the device
against the oracle's FP32 restatement applied to the downloaded REAL
tallies: every normalised flux, error array and image agrees bit for bit,
NaNs included (a peeled Stokes sum of zero gives a NaN error in the
reference too)."""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ipeel", [0, 1])
def test_diskflux_matches_the_oracle_restatement(oracle_mod, ipeel):
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.with_diffusion(model.warm(model.small_2d()))
    n = 20000
    ltot = 3.71
    eng = Engine(m, precision="fp64")
    eng.reset_tallies()
    eng.run(n, ipeel=ipeel)
    raw = eng.download(images=True)
    got = eng.diskflux(n, ltot, ipeel=ipeel, images=True)
    eng.close()
    c = m.config
    ref = oracle_mod.diskflux(raw, n, ltot, c["nmu"], c["nph"], ipeel, bool(c["output_imcube"]))
    assert (raw["nums"] > 1).any()
    for k, v in ref.items():
        assert np.array_equal(got[k], v, equal_nan=True), k
    # unnormalised arrays pass through: counts, and the peeled arrays without ipeel
    assert np.array_equal(got["nabs"], raw["nabs"])
    if ipeel == 0:
        assert np.array_equal(got["ti"], raw["ti"])
    else:
        assert np.isfinite(got["ti2"][raw["numt"] > 1]).any()
    # the SED normalisation: sum of si over the whole SED times rnorm is the raw sum
    rnorm = np.float32(n / c["nmu"] / c["nph"] / ltot)
    assert np.isclose(got["si"].astype(np.float64).sum() * rnorm, raw["si"].astype(np.float64).sum(), rtol=1e-5)
