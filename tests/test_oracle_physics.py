"""Known-answer tests of the CPU oracle (the checker the GPU tests use)."""
import numpy as np
import pytest

from src3_mpi_cfitsio_b200 import abi, model


def _empty(m):
    m.grid["densarr"] = np.zeros_like(m.grid["densarr"])
    return m


def test_unobscured_star(oracle_mod):
    """Empty grid: every packet escapes once; the direct peel-off weight
    4 mu (limb=0, newdisktherm_5_fuv.f90:382-390) integrates to one packet
    per packet for every inclination."""
    m = _empty(model.small_2d())
    b = abi.Bundle(m)
    n = 20000
    tal, log = oracle_mod.run(b, n, threads=4, nlog=n)
    L = abi.packet_log_to_numpy(log)
    assert (L["status"] == 0).all()
    assert (L["nscat"] == 0).all() and (L["nabs"] == 0).all()
    s = tal.scalars()
    assert s["flux"] == n and s["tot"] == 0
    nums = tal.shaped("nums")
    assert nums[..., 0].sum() == n            # total component
    assert nums[..., 1].sum() == n            # stellar origin (1 + i_orig)
    assert nums[..., 5].sum() == n            # direct (5 + i_inter)
    ti = tal.shaped("ti")[:, :, 0, 0].sum(axis=0)   # per inclination
    assert np.allclose(ti / n, 1.0, atol=0.03), ti / n


def test_planck_spectrum(oracle_mod):
    """bbfreq samples B_nu(T*) (random.f90:197-225): the exit frequencies of
    an empty grid follow the Planck distribution."""
    m = _empty(model.small_2d())
    b = abi.Bundle(m)
    n = 40000
    _, log = oracle_mod.run(b, n, ipeel=0, threads=4, nlog=n)
    x = abi.packet_log_to_numpy(log)["nub"] / m.config["tstar"]   # h nu / k T
    # mean of x under x^3/(e^x-1): 4 zeta(5)/zeta(4) = 3.8322 (sd 2.2 -> 4 sigma = 0.045)
    assert abs(x.mean() - 3.8322) < 0.045
    # fraction below x=1: 15/pi^4 * int_0^1 x^3/(e^x-1) dx = 0.034618
    assert abs((x < 1.0).mean() - 0.034618) < 0.004


def test_packet_conservation(oracle_mod, small_model):
    """Each packet ends exactly once: exited + killed + dropped = np."""
    b = abi.Bundle(small_model)
    n = 3000
    tal, log = oracle_mod.run(b, n, threads=4, nlog=n)
    c = tal.counters()
    st = abi.packet_log_to_numpy(log)["status"]
    assert c["packets"] == n
    assert c["exited"] + c["killed"] + c["geom_fail"] + (st == 2).sum() == n
    assert c["geom_fail"] == 0
    # SED: every exited packet lands in the total component once
    assert tal.shaped("nums")[..., 0].sum() == c["exited"]


def test_polarisation_bound(oracle_mod, small_model):
    """Q^2+U^2+V^2 <= I^2 after scattering (propagate_5_fuv.f90:92-109)."""
    b = abi.Bundle(small_model)
    n = 3000
    _, log = oracle_mod.run(b, n, ipeel=0, threads=4, nlog=n)
    L = abi.packet_log_to_numpy(log)
    p2 = L["sqp"] ** 2 + L["sup"] ** 2 + L["svp"] ** 2
    assert np.all(p2 <= L["sip"] ** 2 * (1 + 1e-9))
    assert (L["nscat"] > 0).sum() > 10


def test_accretion_packets_leave_the_disk(oracle_mod):
    """Disk-accretion packets (initpacc_4.f90) with the diffusion treatment:
    each is emitted once by a thermal component (one dbig and one nabs
    count per packet on top of the absorptions), reemitted thermally, and
    leaves the grid."""
    m = model.with_diffusion(model.warm(model.small_2d()))
    m.config["accfrac"] = 0.25
    n, npacc = 2000, 500
    tal, log = oracle_mod.run(abi.Bundle(m), n, ipeel=0, threads=2, nlog=n)
    L = abi.packet_log_to_numpy(log)
    acc = L["iphot"] < npacc
    assert acc.sum() == npacc - 1
    assert (L["status"] == 0).all()
    assert set(np.unique(L["i_orig"][acc])) <= {2, 3, 4}
    absorptions = int(L["nabs"].sum())
    assert tal["dbig"].sum() == absorptions + npacc - 1


def test_tabulated_matrix_reproduces_the_analytic_law(oracle_mod):
    """stokes6 with tables generated from the dustmat law (model.with_mueller)
    scatters like the analytic stokes: the same flux, scatterings and linear
    polarisation within the Monte Carlo error, and no circular polarisation
    without S34."""
    n = 20000
    out = {}
    for name, m in (("analytic", model.warm(model.small_2d())),
                    ("table", model.with_mueller(model.warm(model.small_2d())))):
        tal, log = oracle_mod.run(abi.Bundle(m), n, ipeel=1, threads=4, nlog=n)
        out[name] = (tal, abi.packet_log_to_numpy(log))
    (ta, la), (tt, lt) = out["analytic"], out["table"]
    assert abs(lt["nscat"].sum() - la["nscat"].sum()) <= 0.03 * la["nscat"].sum()
    for k in ("ti", "nums"):
        x, y = ta[k].astype(np.float64).sum(), tt[k].astype(np.float64).sum()
        assert abs(y - x) <= 0.01 * abs(x), k
    assert abs(tt["tq"].astype(np.float64).sum() - ta["tq"].astype(np.float64).sum()) <= \
        0.2 * abs(ta["tq"].astype(np.float64).sum()) + 0.002 * ta["ti"].astype(np.float64).sum()
    assert tt["tv"].sum() == 0.0 and (lt["svp"] == 0.0).all()


def test_tabulated_s34_makes_circular_polarisation_within_the_bound(oracle_mod):
    m = model.with_mueller(model.warm(model.small_2d()), s34_frac=0.8)
    n = 10000
    tal, log = oracle_mod.run(abi.Bundle(m), n, ipeel=1, threads=4, nlog=n)
    L = abi.packet_log_to_numpy(log)
    scattered = L["nscat"] > 0
    assert np.abs(L["svp"][scattered]).max() > 1e-3
    pol = np.sqrt(L["sqp"] ** 2 + L["sup"] ** 2 + L["svp"] ** 2)
    assert (pol <= L["sip"] * (1.0 + 1e-9) + 1e-12).all()
    assert np.abs(tal["tv"].astype(np.float64)).sum() > 0.0


def _adjoint_weights(m):
    c = m.config
    lam = np.zeros((c["nfreq"], c["npeel"], c["nap"], 8))
    lam[:, :, :, 0] = np.linspace(0.5, 1.5, c["nfreq"])[:, None, None]   # total component, graded in frequency
    return lam.ravel(order="F")


def test_oracle_adjoint_matches_central_differences(oracle_mod):
    """Path-replay adjoint (oracle restatement) against central finite
    differences with common random numbers: scaling one density component
    everywhere by exp(+-eps) changes L by 2 eps * sum(grad[:, component]).
    The envelope and cavity components are checked (their estimators
    converge at 1e5 packets; the optically thick disk needs far more).
    Measured on this model at 1e6 packets and three seeds, the two sides
    agree within 3 %."""
    import copy
    base = model.with_diffusion(model.warm(model.small_2d()))
    c = base.config
    lam = np.zeros((c["nfreq"], c["npeel"], c["nap"], 8))
    lam[:, :, :, 0] = 1.0                     # the total peeled flux
    lam = lam.ravel(order="F")
    ncell = c["nrg"] * c["ntg"] * c["npg"]
    n, eps = 300000, 0.05                     # ~3 % Monte Carlo noise on either side at this size
    g, L = oracle_mod.adjoint(abi.Bundle(base), n, lam, threads=8)
    G = g.reshape((ncell, 10), order="F")
    dens = base.grid["densarr"].reshape((ncell, 10), order="F")
    checked = 0
    for comp in (2, 3):                       # 0-based columns: component ids 3 and 4
        if not (dens[:, comp] > 0).any():
            continue
        vals = []
        for sgn in (1, -1):
            mm = copy.deepcopy(base)
            d = dens.copy()
            d[:, comp] *= np.exp(sgn * eps)
            mm.grid["densarr"] = d.ravel(order="F")
            vals.append(oracle_mod.adjoint(abi.Bundle(mm), n, lam, threads=8)[1])
        fd = (vals[0] - vals[1]) / (2 * eps)
        adj = G[:, comp].sum()
        assert abs(adj - fd) <= 0.1 * abs(fd), (comp + 1, adj, fd)
        checked += 1
    assert checked == 2 and L > 0


def test_disk_law_log_derivatives():
    """Chain-rule factors of the disk parameters: rho_disk is proportional
    to Mdisk; d log rho/d log h100 = z^2/h^2 - 1 (the scale height and the
    normalisation); with_disk_params changes the disk cells only."""
    m = model.small_2d()
    w = m.w
    d = model.disk_log_derivatives(m)
    on = d["massd"] != 0
    assert on.sum() > 10 and np.allclose(d["massd"][on], 1.0, atol=1e-6)
    autors = 214.94 / w.rstar
    r = m.grid["rarr"]; t = m.grid["thetarr"]
    rad = (0.5 * (r[:-1] + r[1:]))[:, None]
    th = (0.5 * (t[:-1] + t[1:]))[None, :]
    wcyl, z = rad * np.sin(th), rad * np.abs(np.cos(th))
    h = w.h100_au * autors / (100.0 * autors) ** w.b_exp * wcyl ** w.b_exp
    expect = (z / h) ** 2 - 1.0
    assert np.allclose(d["h100_au"][on], expect[on], rtol=1e-5, atol=1e-6)
    mm = model.with_disk_params(m, massd=2.0 * w.massd)
    a = m.grid["densarr"].reshape(-1, 10, order="F")
    b = mm.grid["densarr"].reshape(-1, 10, order="F")
    assert np.allclose(b[:, 1], 2.0 * a[:, 1], rtol=1e-12) and np.array_equal(b[:, 2:], a[:, 2:])


def _gray_dust(nl=100, kap=2.0, alb=0.25):
    nud = np.logspace(2, -4, nl)
    return nud, np.full(nl, kap), np.full(nl, alb)


def test_setemiss_oracle_gray_dust_is_the_planck_integral():
    """setemiss restatement (dust_5.f90:507-699) for a gray absorber: the
    Planck mean is (1-albedo) kappa times the normalised Planck integral up to
    x = 32, the Rosseland mean is kappa, and the cumulative table is the
    normalised Planck integral, all to the qsimp tolerance (1e-5) and the
    reference's 7-digit 15/pi^4 and A&S expm1."""
    from scipy import integrate
    from oracle import oracle as O
    nud, kd, ad = _gray_dust()
    r = O.setemiss(nud, kd, ad, [nud.size], threads=4)
    assert r["qsimp_misses"] == 0
    norm = 0.1539897
    F = lambda x: norm * x ** 3 / np.expm1(x)
    dF = lambda x: norm * x ** 4 * np.exp(x) / (4.0 * np.expm1(x) ** 2)
    tot = integrate.quad(F, 0, 32, epsabs=0, epsrel=1e-13, limit=200)[0]
    dtot = integrate.quad(dF, 0, 32, epsabs=0, epsrel=1e-13, limit=200)[0]
    assert np.allclose(r["kappap"], 0.75 * 2.0 * tot, rtol=1e-6, atol=0)
    assert np.allclose(r["kappar"], 2.0 / dtot, rtol=1e-6, atol=0)
    ki = r["kapint"].reshape((500, 513), order="F")
    xs = r["nuint"][[10, 64, 200, 400]]
    cum = np.array([integrate.quad(F, 0, x, epsabs=0, epsrel=1e-13)[0] for x in xs]) / tot
    assert np.allclose(ki[250, [10, 64, 200, 400]], cum, rtol=2e-5, atol=0)
    assert np.all(np.diff(ki, axis=1) >= 0) and np.all(ki[:, -1] == 1.0)


def test_setemiss_oracle_agrees_with_an_independent_quadrature():
    """The reference's algorithm (qsimp per interval, opacity and albedo
    interpolated separately) against the model generator's 12-point
    Gauss-Legendre tables of the same dust law."""
    from oracle import oracle as O
    m = model.small_2d()
    t = m.tables
    r = O.setemiss(t["nudust"], t["kappad"], t["adust"], t["nlambda"], threads=4)
    assert np.array_equal(r["lTint"], t["lTint"]) and np.array_equal(r["nuint"], t["nuint"])
    assert np.abs(r["kappap"] / t["kappap"] - 1).max() < 1e-3
    assert np.abs(r["kappar"] / t["kappar"] - 1).max() < 1e-4
    assert np.abs(r["kapint"] - t["kapint"]).max() < 1e-3


def test_setemiss_oracle_smooths_gas_planck_means():
    """Species above ndg (gas opacities) get two passes of the 21-point box
    average of the Planck mean with the window shrinking at the ends
    (dust_5.f90:623-663); dust species and the other tables are unchanged."""
    from oracle import oracle as O
    nl = 60
    nud = np.logspace(2, -4, nl)
    lam = 1.2398 / nud
    cols = [np.stack([nud, 3.0 * lam ** -1.5, 0.5 / (1 + lam)]),
            np.stack([nud, 1.0 + np.sin(np.log(lam)) ** 2, np.full(nl, 0.1)])]
    nudust = np.concatenate([c[0] for c in cols])
    kd = np.concatenate([c[1] for c in cols])
    ad = np.concatenate([c[2] for c in cols])
    a = O.setemiss(nudust, kd, ad, [nl, nl], threads=2)
    b = O.setemiss(nudust, kd, ad, [nl, nl], ndg=1, threads=2)
    nT = 500
    assert np.array_equal(a["kapint"], b["kapint"]) and np.array_equal(a["kappar"], b["kappar"])
    assert np.array_equal(a["kappap"][:nT], b["kappap"][:nT])
    kp = a["kappap"][nT:].copy()
    for _ in range(2):
        out = np.empty(nT)
        for i in range(1, nT + 1):
            lo, hi = (i - 10, i + 10) if 10 < i <= nT - 10 else ((1, 2 * i + 1) if i <= 10 else (2 * i - nT, nT))
            out[i - 1] = kp[lo - 1:hi].sum() / (hi - lo + 1)
        kp = out
    assert np.allclose(b["kappap"][nT:], kp, rtol=1e-13, atol=0)


def test_isrf_packets_sample_the_table_and_are_not_binned_unscattered(oracle_mod):
    """External illumination (initpout.f90 + rep_isrf.f90): in an empty grid
    every packet crosses unscattered, so its exit frequency is its emitted
    one and nothing is binned (unscattered external light is the sky
    background, not part of the SED).  The frequencies follow the table:
    mapped back through its log-log interpolation they are uniform on
    (cdf_2, 1)."""
    m = model.with_isrf(model.warm(model.small_2d()), 1.0)
    m.grid["densarr"] = np.zeros_like(m.grid["densarr"])
    n = 20000
    tal, lo = oracle_mod.run(abi.Bundle(m), n, ipeel=1, nlog=n, threads=4)
    g = abi.packet_log_to_numpy(lo)
    c = tal.counters()
    assert c["packets"] == n and c["exited"] == n and c["interactions"] == 0
    assert np.all(g["i_orig"] == 5) and np.all(g["nscat"] == 0)
    assert tal["si"].sum() == 0 and tal["ti"].sum() == 0 and tal["image_m_i"].sum() == 0
    t = m.tables["isrf"]
    k = t.size // 3
    cdf, lcdf, lfr = t[:k], t[k:2 * k], t[2 * k:]
    lnu = np.log10(g["nub"])
    sel = lnu >= lfr[1]
    i = np.clip(np.searchsorted(lfr[1:], lnu[sel], side="right"), 1, k - 2)    # rows i..i+1 (0-based, >= 1)
    x = 10.0 ** (lcdf[i] + (lnu[sel] - lfr[i]) / (lfr[i + 1] - lfr[i]) * (lcdf[i + 1] - lcdf[i]))
    u = np.sort((x - cdf[1]) / (1.0 - cdf[1]))
    ks = np.max(np.abs(u - (np.arange(1, u.size + 1) - 0.5) / u.size))
    assert sel.mean() > 0.99 and ks < 1.63 / np.sqrt(u.size) + 1e-3


def test_sweep_workloads_follow_the_configured_ranges():
    """The batched sweep's models: nr 50-200, ntheta 49-199 (odd wall count),
    nphi 1-32 cells, Mdisk in 1e-4..0.1 Msun, Mdot in 1e-7..1e-5 Msun/yr,
    cavity 5-40 deg, 60-140 wavelengths; seeded, so repeatable."""
    ws = model.batch_workloads(64)
    assert len(ws) == 64
    for w in ws:
        assert 50 <= w.nrg - 1 <= 200 and 49 <= w.ntg <= 199 and w.ntg % 2 == 1 and 1 <= w.npg - 1 <= 32
        assert 1e-4 <= w.massd <= 0.1 and 1e-7 <= w.rate <= 1e-5 and 5.0 <= w.thet1_deg <= 40.0
        assert 60 <= w.nlambda <= 140
    again = model.batch_workloads(64)
    assert all(a == b for a, b in zip(ws, again))
    assert len({(w.nrg, w.ntg, w.npg) for w in ws}) > 50            # uneven grids


def test_isrf_table_has_the_reference_layout():
    """isrf_table: a normalised non-decreasing cdf over ascending
    frequencies, log10 columns consistent with it, and the first row as
    isrf_cdf.f90 leaves it (cdf 0, log cdf -99, log nu 0)."""
    t = model.isrf_table()
    k = t.size // 3
    cdf, lcdf, lfr = t[:k], t[k:2 * k], t[2 * k:]
    assert k == 200 and cdf[0] == 0.0 and lcdf[0] == -99.0 and lfr[0] == 0.0
    assert np.all(np.diff(cdf) >= 0) and cdf[-1] == 1.0
    assert np.allclose(lcdf[1:], np.log10(cdf[1:])) and np.all(np.diff(lfr[1:]) > 0)
    # wavelengths lmin (lmax/lmin)^(i/200), i = 1..200 (the loop of
    # isrf_cdf.f90 starts at i = 1), so the top frequency sits one step
    # below 1.2398/lmin eV
    top = 1.2398 / (0.0912 * (1000.0 / 0.0912) ** (1.0 / 200))
    assert abs(10 ** lfr[-1] / top - 1.0) < 1e-9 and 10 ** lfr[1] > 1.2398 / 1000.0


def test_tfinal_velocity_field_reduces_to_the_gas_at_rest(oracle_mod):
    """With a velocity field of zeros the passes of tfinal give the result of
    a gas at rest bit for bit (the adiabatic and advective terms are exact
    zeros); the envelope's infall field changes the temperature of envelope
    cells only, by well under a percent."""
    import copy
    from src3_mpi_cfitsio_b200 import abi, model
    m = model.reference_2d_converged()
    mv = model.with_velocities(copy.deepcopy(m))
    mz = copy.deepcopy(mv)
    for k in ("vrarr", "vthetarr", "divvarr"):
        mz.grid[k] = np.zeros_like(mz.grid[k])
    n = 100000
    tal, _ = oracle_mod.run(abi.Bundle(m), n, ipeel=0, images=False)
    env = (m.dens4()[..., 2] > 0).ravel(order="F")
    for it in (2, 5):
        a, _ = oracle_mod.tfinal(abi.Bundle(m), tal["dtauabs"], n, it, m.grid["tdust"])
        b, _ = oracle_mod.tfinal(abi.Bundle(mz), tal["dtauabs"], n, it, m.grid["tdust"])
        c, _ = oracle_mod.tfinal(abi.Bundle(mv), tal["dtauabs"], n, it, m.grid["tdust"])
        assert np.array_equal(a, b)
        rel = np.abs(c / a - 1.0)
        assert rel[~env].max() == 0.0
        assert 1e-5 < rel[env].max() < 1e-2


def test_oracle_adjoint_control_variate(oracle_mod):
    """The replay's control variate (each segment's score weighted by A - B):
    B = 0 everywhere reproduces the plain replay exactly (the extra packets
    without peel-off records then add nothing), and a learning replay
    counts one segment start per packet plus one per interaction."""
    m = model.with_diffusion(model.warm(model.small_2d()))
    b = abi.Bundle(m)
    lam = _adjoint_weights(m)
    c = m.config
    ncell = c["nrg"] * c["ntg"] * c["npg"]
    n = 3000
    g0, L0 = oracle_mod.adjoint(b, n, lam, threads=4)
    for nfb in (5, -5):                       # -5: five frequency bins x four direction classes
        nv = ncell * 5 * (4 if nfb < 0 else 1)
        g1, L1, _, _ = oracle_mod.adjoint_cv(b, n, lam, vtab=np.zeros(nv), nfb=nfb, threads=4)
        assert abs(L1 - L0) <= 1e-12 * L0      # threads take packets in any order
        assert np.allclose(g1, g0, rtol=1e-12, atol=1e-12 * np.abs(g0).max())
    # without diffusion cells the replay's paths are those of an ordinary run
    b = abi.Bundle(model.warm(model.small_2d()))
    _, L2, vs, vc = oracle_mod.adjoint_cv(b, n, lam, nfb=-5, learn=True, threads=4)
    assert L2 > 0
    _, log = oracle_mod.run(b, n, ipeel=0, nlog=n, threads=4)
    events = abi.packet_log_to_numpy(log)
    segments = n + int(events["nscat"].sum() + events["nabs"].sum())
    assert vc.sum() == segments
    assert (vc >= 0).all() and np.isfinite(vs).all() and vs.sum() > 0


def test_rep_draine_samples_the_draine_spectrum(oracle_mod):
    """rep_draine (oracle restatement) draws frequencies whose distribution
    is the row's cumulative spectrum: the fraction of draws below each
    column frequency matches cdf_d at that column (Kolmogorov distance of
    2e5 draws below 5e-3, where the sampling error is ~2e-3); rows of
    higher intensity ratio emit bluer."""
    m = model.with_small_grains(model.warm(model.small_2d()))
    b = abi.Bundle(m)
    ne, nd = m.tables["nemit"], m.tables["ndraine"]
    t = m.tables["draine"]
    cdf = t[:ne * nd].reshape((ne, nd), order="F")
    freq = 10.0 ** t[2 * ne * nd:]
    medians = []
    for im in (1, 2, 9, 18):
        nu = np.sort(oracle_mod.rep_draine(b, im, 200000))
        assert np.isfinite(nu).all() and (nu > 0).all()
        emp = np.searchsorted(nu, freq[1:], side="right") / nu.size
        assert np.abs(emp - cdf[im - 1, 1:]).max() < 5e-3, im
        medians.append(np.median(nu))
    assert medians[-1] > medians[0]


def test_small_grains_reemit_in_cells_without_thermal_dust(oracle_mod):
    """With small grains in the disk and envelope and a small-grain-only
    cavity, absorptions by small grains (dsg) occur only in cells without
    thermal dust (select_dust's one-thermal-component rule), every packet
    is accounted for, and the first and a later iteration (Draine rows 2
    and 1) both run."""
    m = model.with_small_grains(model.warm(model.small_2d()))
    d = m.dens4()
    thermal = (d[..., [0, 1, 2, 3, 8, 9]] > 0).any(axis=-1)
    n = 20000
    for it in (1, 2):
        tal, _ = oracle_mod.run(abi.Bundle(m), n, ipeel=0, iteration=it, threads=4)
        dsg = tal["dsg"].reshape(d.shape[:3], order="F")
        assert dsg.sum() > 0 and dsg[thermal].sum() == 0
        c = tal.counters()
        assert c["packets"] == n and c["exited"] + c["killed"] + c["geom_fail"] == n
