"""Nested multi-wavelength images (output_imsparse; peeloff_3d_2_test.f90:
302-309, type_nested_image.f90:75-101, math_binning.f90): the oracle's
binning checked on the CPU for flux conservation and level geometry, and the
engine's binning on every peel-off path against the oracle."""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model


@pytest.fixture(scope="module")
def nested():
    return model.with_nested_images(model.warm(model.small_2d()))


def test_levels_follow_find_levels():
    lev = model.nested_levels(1000.0, 10.0, 4)
    assert lev.dtype == np.float32
    assert lev.size == int(np.ceil(np.log10(100.0) / np.log10(4.0))) + 1
    assert lev[-1] == np.float32(1000.0)
    assert np.all(lev[1:] / lev[:-1] == np.float32(4.0))


def test_oracle_nested_images_hold_the_image_flux(nested, oracle_mod):
    """The nested images cover the same square as the image cube (half size
    rmaxi), so their Stokes I adds up to the cube's, up to the peel-offs whose
    frequency falls outside the SED range (the cube clamps those to its end
    bins, the nested images drop them)."""
    tal, _ = oracle_mod.run(abi.Bundle(nested), 20000, ipeel=1, threads=8)
    cube = tal["image_m_i"].astype(np.float64).sum()
    ms = tal["image_ms_i"].astype(np.float64).sum()
    assert cube > 0
    assert abs(ms - cube) < 1e-3 * cube


def test_oracle_nested_levels_are_annuli(nested, oracle_mod):
    """A peel-off goes to the smallest level whose half size exceeds
    max(|x|,|y|): every lit pixel of level l >= 2 lies outside level l-1's
    square (within one pixel), and the innermost level is used."""
    tal, _ = oracle_mod.run(abi.Bundle(nested), 20000, ipeel=1, threads=8)
    ims = tal.shaped("image_ms_i").astype(np.float64)          # [dim, dim, nnu, nlev, npeel]
    lev = nested.tables["sparse_levels"].astype(np.float64)
    dim = nested.config["sparse_dim"]
    assert ims[:, :, :, 0, :].sum() > 0
    for l in range(1, lev.size):
        lit = np.argwhere(ims[:, :, :, l, :].sum(axis=(2, 3)) != 0)
        if lit.size == 0:
            continue
        h = lev[l]
        px = 2.0 * h / dim
        xc = -h + (lit[:, 0] + 0.5) * px
        yc = -h + (lit[:, 1] + 0.5) * px
        assert (np.maximum(np.abs(xc), np.abs(yc)) >= lev[l - 1] - px).all(), l


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", ["wave", "warp", "packet"])
def test_nested_images_match_the_oracle(nested, oracle_mod, schedule):
    from src3_mpi_cfitsio_b200.engine import Engine
    n = 20000
    eng = Engine(nested, precision="fp64")
    eng.set_schedule(schedule)
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    g = eng.download(images=True)
    raw_flux = eng.diskflux(n, 3.71, ipeel=1, images=True)
    eng.close()
    o, _ = oracle_mod.run(abi.Bundle(nested), n, ipeel=1, threads=8)
    for k in abi.IMGS:
        a, b = g[k].astype(np.float64), o[k].astype(np.float64)
        scale = max(np.abs(b).max(), 1e-300)
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6 * scale), k
        assert np.array_equal(raw_flux[k], g[k]), k          # diskflux leaves them as binned
    assert o["image_ms_i"].sum() > 0
