"""Filter-band images (output_imfilt, peeloff_3d_2_test.f90:242-285): the
oracle's binning checked on the CPU against what the images must hold, and
the engine's binning (job-queue peel-offs of the wavefront schedule, inline
peel-offs of the warp schedule, the per-thread kernel) against the oracle on
the same packets, with the diskflux normalisation (flux_test.f90:64-73)."""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model


def _flat_filter(m):
    """One filter spanning every frequency of the SED grid with response 1:
    its image must be the image cube summed over frequency."""
    c = m.config
    numin, numax = c["numin"], c["numin"] * np.exp(c["lnurat"])
    f = np.geomspace(0.5 * numin / 1.2398 * 2.9979e14, 2.0 * numax / 1.2398 * 2.9979e14, 40)
    m.tables["nwfilt"] = np.array([f.size + 1], np.int32)
    m.tables["filtwave"] = f
    m.tables["filtphi"] = np.ones_like(f)
    m.config.update(output_imfilt=1, nfilt=1, nwfiltmax=f.size)
    return m


def test_oracle_flat_filter_image_is_the_summed_cube(oracle_mod):
    m = _flat_filter(model.warm(model.small_2d()))
    tal, _ = oracle_mod.run(abi.Bundle(m), 20000, ipeel=1, threads=8)
    cube = tal.shaped("image_m_i").astype(np.float64).sum(axis=3)
    band = tal.shaped("image_b_i")[..., 0].astype(np.float64)
    assert cube.sum() > 0
    assert np.allclose(band, cube, rtol=1e-5, atol=1e-6 * cube.max())
    for s in ("q", "u"):
        c2 = tal.shaped(f"image_m_{s}").astype(np.float64).sum(axis=3)
        assert np.allclose(tal.shaped(f"image_b_{s}")[..., 0], c2, rtol=1e-5, atol=1e-6 * np.abs(c2).max())


def test_oracle_origin_images_add_up_to_stokes_i(oracle_mod):
    """Every packet has an origin 1..4 (star, disk, envelope, outflow), so the
    four origin images sum to the Stokes I image of each band."""
    m = model.with_filters(model.warm(model.small_2d()))
    tal, _ = oracle_mod.run(abi.Bundle(m), 20000, ipeel=1, threads=8)
    i = tal["image_b_i"].astype(np.float64)
    parts = sum(tal[k].astype(np.float64) for k in ("image_b_d", "image_b_s", "image_b_e", "image_b_o"))
    assert i.sum() > 0
    assert np.allclose(parts, i, rtol=1e-5, atol=1e-6 * i.max())
    for k in ("image_b_d", "image_b_s", "image_b_e"):
        assert tal[k].sum() > 0, k


def test_filter_curves_are_ascending_and_normalised():
    """The generator's curves follow filt_nu.f90: frequency ascending within
    each curve and the response's trapezoidal integral over frequency 1."""
    nwfilt, fw, fp = model.filter_table()
    nmax = fw.size // nwfilt.size
    FW = fw.reshape((nmax, nwfilt.size), order="F")
    FP = fp.reshape((nmax, nwfilt.size), order="F")
    for b in range(nwfilt.size):
        n = nwfilt[b] - 1
        f, p = FW[:n, b], FP[:n, b]
        assert (np.diff(f) > 0).all()
        assert np.isclose(np.sum(0.5 * (p[1:] + p[:-1]) * np.diff(f)), 1.0, rtol=1e-12)


@pytest.mark.gpu
def test_upload_refuses_a_descending_filter():
    from src3_mpi_cfitsio_b200.engine import Engine, MCRTError
    m = model.with_filters(model.warm(model.small_2d()))
    nmax, nf = m.config["nwfiltmax"], m.config["nfilt"]
    fw = m.tables["filtwave"].reshape((nmax, nf), order="F").copy()
    n = m.tables["nwfilt"][0] - 1
    fw[:n, 0] = fw[:n, 0][::-1]
    m.tables["filtwave"] = np.asfortranarray(fw).ravel(order="F")
    with pytest.raises(MCRTError) as e:
        Engine(m, precision="fp64")
    assert e.value.code == 1


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", ["wave", "warp", "packet"])
def test_filter_images_match_the_oracle(oracle_mod, schedule):
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.with_filters(model.warm(model.small_2d()))
    n = 20000
    eng = Engine(m, precision="fp64")
    eng.set_schedule(schedule)
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    g = eng.download(images=True)
    eng.close()
    o, _ = oracle_mod.run(abi.Bundle(m), n, ipeel=1, threads=8)
    for k in abi.IMGB:
        a, b = g[k].astype(np.float64), o[k].astype(np.float64)
        scale = max(np.abs(b).max(), 1e-300)
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6 * scale), k
    assert o["image_b_i"].sum() > 0


@pytest.mark.gpu
def test_filter_images_are_normalised_by_diskflux(oracle_mod):
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.with_filters(model.warm(model.small_2d()))
    n = 20000
    ltot = 3.71
    eng = Engine(m, precision="fp64")
    eng.reset_tallies()
    eng.run(n, ipeel=1)
    raw = eng.download(images=True)
    got = eng.diskflux(n, ltot, ipeel=1, images=True)
    eng.close()
    inorm = np.float32(n / ltot)
    for k in abi.IMGB:
        assert np.array_equal(got[k], (raw[k] / inorm).astype(np.float32)), k
