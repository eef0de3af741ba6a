"""Synthetic young-star models in the reference's array layout.

The reference builds its model on the host before every call of ``disk``:
walls and densities in ``gridset`` (gridset_5_model13new.f90), dust tables in
``dustinit``/``setemiss`` (dust_5.f90:345-699) and the stellar CDF in
``atmosinit`` (starbarb_2.f90:3-122).  Those routines stay outside the packet
engine; this module produces the same arrays from the analytic recipes the
benchmark workloads name, so that the engine and its oracle can be driven
without the reference's missing parameter files:

* walls: wall 1 is the stellar surface, wall 2 the dust inner radius, then
  log-spaced walls to ``rmax``; theta walls keep the reference convention of an
  odd wall count with a theta=90 deg wall flagged by ``tan2arr=-1``
  (gridset_5_model13new.f90:722-750, thetaface.f90:33-53);
* disk: Whitney flared disk normalised to its mass (setup_wave.f90:60-88),
  rho = rho0 (1-sqrt(R*/w)) (R*/w)^a exp(-z^2/2h^2), h = z1 w^b;
* envelope: Ulrich rotating infall (densenv.f90:37-43, envset.f90:157-160,
  zerod.f90) with the ambient floor; polynomial bipolar cavity
  (densenv.f90:76-90, envset.f90:182-189); disk cells clear the envelope and
  cavity components (gridset_5_model13new.f90:1217-1224);
* dust: kappa = kappa0 (lambda/1um)^-1.5 on 100 log wavelengths 0.1-3000 um,
  albedo 0.5->0 and g 0.6->0 linear in log lambda, pmax 0.5; normalised to
  0.55 um like dustinit (dust_5.f90:457-464); kapint/kappap/kappar follow the
  setemiss integrals (dust_5.f90:507-699) with Gauss-Legendre quadrature in
  place of Numerical Recipes' qsimp;
* star: Planck atmosphere CDF as atmosinit builds it with CPLANCKST=YES.

All arrays are returned flattened in Fortran (column-major) order.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

# constants.f90
PI = 3.1415926535897932384626433
R2P = 2.0 * PI
RSOL = 6.9598e10
MSOL = 1.989e33
GN = 6.67428e-8
SIGT = 5.670400e-5
KB = 1.3806503e-16
MH = 1.67262158e-24

NDG2 = 10
NO = 8


@dataclasses.dataclass
class Workload:
    """Parameters of one model; defaults are the 2-D reference workload."""
    # grid (wall counts, Fortran nrg/ntg/npg)
    nrg: int = 101
    ntg: int = 99
    npg: int = 2
    # star
    rstar: float = 2.0            # Rsun
    tstar_k: float = 4000.0       # K
    # geometry [AU]
    rddust_au: float = 0.1
    rmax_au: float = 5000.0
    rmaxd_au: float = 200.0
    # disk
    massd: float = 0.01           # Msun
    a_exp: float = 2.25
    b_exp: float = 1.25
    h100_au: float = 10.0
    # envelope
    rate: float = 1.0e-6          # Msun/yr
    rc_au: float = 100.0
    massc: float = 0.5            # Msun
    rhoamb: float = 1.67e-20
    # cavity
    thet1_deg: float = 20.0
    ex1: float = 1.5
    rhoconst1: float = 1.67e-19
    # dust law
    kappa0: float = 100.0         # cm^2/g at 1 um
    nlambda: int = 100
    # SEDs / images
    nfreq: int = 100
    nmu: int = 10
    nph: int = 1
    nap: int = 1
    npeel: int = 10
    nxhst: int = 101
    rmaxi_au: float = 5000.0
    aperture_au: float = 5000.0
    # theta-wall clustering toward the equator
    theta_power: float = 2.0
    # inner-rim refinement (gridset_5_model13new.f90:437-493): number of walls
    # spent between the dust rim and rim_top_au, the first cell holding a
    # midplane Rosseland optical depth of rim_tau
    rim_walls: int = 20
    rim_top_au: float = 0.15
    rim_tau: float = 0.5
    # multiplicative clump field (3-D fractal models); None for smooth models
    clump_seed: int | None = None
    clump_dim: float = 2.6
    clump_mass_frac: float = 0.5


class Model:
    """A complete engine input: config scalars plus grid and table arrays."""

    def __init__(self, w: Workload):
        self.w = w
        self.config: dict = {}
        self.grid: dict = {}
        self.tables: dict = {}
        self._build()

    # ------------------------------------------------------------------ walls
    def _walls(self):
        w = self.w
        autors = 214.94 / w.rstar                      # setup.f90:45
        rddust = w.rddust_au * autors
        rmax = w.rmax_au * autors
        nrg, ntg, npg = w.nrg, w.ntg, w.npg
        if ntg % 2 == 0:
            raise ValueError("ntg must be odd (theta=90 wall), grid_mod_5.f90:6")
        rarr = np.empty(nrg)
        rarr[0] = 1.0                                  # stellar surface
        rarr[1] = rddust
        nf = self._rim_walls(autors, rddust) if (w.rim_walls > 0 and w.massd > 0) else np.empty(0)
        nfw = nf.size
        rarr[2:2 + nfw] = nf
        r0 = rarr[1 + nfw]
        nlog = nrg - 2 - nfw
        rarr[2 + nfw:] = r0 * (rmax / r0) ** (np.arange(1, nlog + 1) / nlog)
        rarr[-1] = rmax
        r2arr = rarr * rarr

        nttmp = (ntg + 1) // 2
        tmpth = 0.5 * PI * (np.arange(nttmp) / (nttmp - 1)) ** w.theta_power
        thetarr = np.empty(ntg)
        for it in range(2, nttmp):                     # gridset_5_model13new.f90:722-725
            thetarr[nttmp + 1 - it - 1] = 0.5 * PI - tmpth[it - 1]
            thetarr[nttmp - 1 + it - 1] = 0.5 * PI + tmpth[it - 1]
        thetarr[0] = 0.0
        thetarr[nttmp - 1] = 0.5 * PI
        thetarr[ntg - 1] = PI
        costarr = np.cos(thetarr)
        sintarr = np.sin(thetarr)
        tan2arr = np.tan(thetarr) ** 2
        costarr[0], sintarr[0], tan2arr[0] = 1.0, 0.0, 0.0
        costarr[-1], sintarr[-1], tan2arr[-1] = -1.0, 0.0, 0.0
        costarr[nttmp - 1], sintarr[nttmp - 1], tan2arr[nttmp - 1] = 0.0, 1.0, -1.0

        dp = R2P / (npg - 1)
        phiarr = dp * np.arange(npg)
        aarr = np.sin(phiarr)
        barr = -np.cos(phiarr)
        return autors, rddust, rmax, rarr, r2arr, thetarr, costarr, sintarr, tan2arr, phiarr, aarr, barr

    def _rim_walls(self, autors, rddust):
        """Walls resolving the optically thick disk rim: the first cell holds a
        midplane Rosseland depth rim_tau (tauw of gridset_5_model13new.f90:437-
        446), then the spacing ratio grows geometrically (rfac <- rfac**gamma,
        :465-469) so that rim_walls walls reach rim_top_au."""
        w = self.w
        rmincgs = w.rstar * RSOL
        rmaxd = w.rmaxd_au * autors
        z1 = w.h100_au * autors / (100.0 * autors) ** w.b_exp
        p = w.b_exp - w.a_exp
        const = R2P ** 1.5 * rmincgs ** 2 * (rmincgs * z1)
        rho0 = w.massd * MSOL / const / (
            1.0 / (p + 2.0) * (rmaxd ** (p + 2.0) - rddust ** (p + 2.0))
            - 1.0 / (p + 1.5) * (rmaxd ** (p + 1.5) - rddust ** (p + 1.5)))
        # Rosseland mean of the dust law at 1400 K relative to V (dust_5.f90:465)
        lam = np.logspace(-1, np.log10(3000.0), 4000)
        x = 1.4388e4 / (lam * 1400.0)
        dB = x ** 5 * np.exp(x) / np.expm1(x) ** 2 / lam ** 0   # dB/dT shape in nu
        nu = 1.0 / lam
        kap = (lam / 0.55) ** -1.5
        wgt = dB * np.gradient(nu)
        chir = np.sum(np.abs(wgt)) / np.sum(np.abs(wgt) / kap)
        kV = w.kappa0 * 0.55 ** -1.5
        # cumulative midplane tau_R from the rim
        rr = rddust * (1.0 + np.logspace(-12, np.log10(w.rim_top_au / w.rddust_au - 1.0 + 1e-12), 20000))
        rho = rho0 * (1.0 - np.sqrt(1.0 / rr)) * rr ** (-w.a_exp)
        dtau = kV * chir * rho * rmincgs
        tau = np.concatenate(([0.0], np.cumsum(0.5 * (dtau[1:] + dtau[:-1]) * np.diff(rr))))
        tau = tau - tau[0]
        r1 = float(np.interp(w.rim_tau, tau, rr))
        rtop = w.rim_top_au * autors
        n = w.rim_walls
        f1 = r1 / rddust
        # rfac_k = f1**(gamma**k); find gamma so that wall n reaches rtop
        def top(gam):
            r = rddust
            f = f1
            for _ in range(n):
                r = r * f
                f = f ** gam
            return r
        lo, hi = 1.0, 3.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if top(mid) > rtop:
                hi = mid
            else:
                lo = mid
        gam = lo
        walls = []
        r, f = rddust, f1
        for _ in range(n):
            r = r * f
            f = f ** gam
            walls.append(r)
        return np.array(walls)

    # ------------------------------------------------------------- densities
    @staticmethod
    def _ulrich_mu0(mu, rx):
        """Root of mu0^3 + (rx-1) mu0 - rx mu = 0 in [0,1] (zerod.f90)."""
        a2 = rx - 1.0
        a3 = -rx * mu
        q = (-3.0 * a2) / 9.0
        r = (27.0 * a3) / 54.0
        q3 = q ** 3
        out = np.empty_like(mu)
        three = (q3 - r * r) >= 0.0
        if np.any(three):
            qq, rr, qq3 = q[three], r[three], q3[three]
            qh = np.sqrt(qq)
            th = np.arccos(np.clip(rr / np.sqrt(qq3), -1.0, 1.0))
            roots = np.stack([-2.0 * qh * np.cos(th / 3.0),
                              -2.0 * qh * np.cos((th + 2.0 * PI) / 3.0),
                              -2.0 * qh * np.cos((th + 4.0 * PI) / 3.0)])
            roots = np.where(roots > 0.0, roots, np.inf)
            out[three] = np.min(roots, axis=0)
        one = ~three
        if np.any(one):
            rr, qq, qq3 = r[one], q[one], q3[one]
            fac = np.sqrt(rr * rr - qq3) + np.abs(rr)
            f3 = fac ** (1.0 / 3.0)
            out[one] = -np.sign(rr) * (f3 + qq / f3)
        return np.clip(out, 1e-12, 1.0)

    def _densities(self, autors, rddust, rmax, rarr, thetarr, npg):
        w = self.w
        nr, nt, npc = w.nrg - 1, w.ntg - 1, npg - 1
        rave = 0.5 * (rarr[:-1] + rarr[1:])
        thave = 0.5 * (thetarr[:-1] + thetarr[1:])
        rad = rave[:, None]
        th = thave[None, :]
        sina = np.sin(th)
        cosa = np.abs(np.cos(th))
        wcyl = rad * sina
        zp = rad * cosa
        rmincgs = w.rstar * RSOL

        # disk (setup.f90:96-99 R100 scale height, setup_wave.f90:60-88)
        rho_d = self._disk_rho(w, autors, rddust, rarr, thetarr)

        # Ulrich envelope (envset.f90:157-160, densenv.f90:37-43)
        rc = w.rc_au * autors
        rdcgs = rc * rmincgs
        cst = 1.0 / 3.15576e7 * math.sqrt(MSOL) / (4.0 * PI) / math.sqrt(GN)
        rhoe0 = cst * w.rate / math.sqrt(w.massc) / rdcgs ** 1.5
        rmine = rddust
        mu = zp / rad
        rx = np.broadcast_to(rad / rc, mu.shape).copy()
        mu0 = self._ulrich_mu0(np.broadcast_to(mu, rx.shape).copy(), rx)
        factor = 1.0 / ((mu / mu0) + 2.0 * mu0 ** 2 / rx)
        rho_e = rhoe0 * rx ** (-1.5) * factor / np.sqrt(1.0 + mu / mu0)
        rho_e = np.where(rad > rmine, np.maximum(rho_e, w.rhoamb), 0.0)

        # polynomial cavity (envset.f90:182-189, densenv.f90:76-90)
        r1max = rmax * math.tan(w.thet1_deg * PI / 180.0)
        c1e = rmax / r1max ** w.ex1
        zup = c1e * wcyl ** w.ex1
        inhole = zp > zup
        rho_c = np.where(inhole & (rad > rmine) & (rad < rmax), w.rhoconst1, 0.0)
        rho_e = np.where(inhole | (rad >= rmax), 0.0, rho_e)

        if w.clump_seed is not None:
            fac = self._clump_field(nr, nt, max(npc, 1))
            rho_e = rho_e[:, :, None] * fac
            rho_c = np.broadcast_to(rho_c[:, :, None], fac.shape)
            rho_d = np.broadcast_to(rho_d[:, :, None], fac.shape)
        else:
            rho_e = np.broadcast_to(rho_e[:, :, None], (nr, nt, npc))
            rho_c = np.broadcast_to(rho_c[:, :, None], (nr, nt, npc))
            rho_d = np.broadcast_to(rho_d[:, :, None], (nr, nt, npc))

        # the disk owns a cell where it is denser than the envelope+cavity gas;
        # there the other components are cleared (gridset_5_model13new.f90:1217-1224)
        rho_d = np.where(rho_d > rho_e + rho_c, rho_d, 0.0)
        disk = rho_d > 0.0
        dens = np.zeros((w.nrg, w.ntg, npg, NDG2))
        dens[:nr, :nt, :npc, 1] = rho_d                      # id 2: disk grains
        dens[:nr, :nt, :npc, 2] = np.where(disk, 0.0, rho_e)  # id 3: envelope
        dens[:nr, :nt, :npc, 3] = np.where(disk, 0.0, rho_c)  # id 4: cavity
        # vcell (gridset_5_model13new.f90:1147-1150)
        dr3 = rarr[1:] ** 3 - rarr[:-1] ** 3
        dcost = np.cos(thetarr[1:]) - np.cos(thetarr[:-1])
        vcell = np.zeros((w.nrg, w.ntg, npg))
        vcell[:nr, :nt, :npc] = (-(dr3[:, None] * dcost[None, :]) * (R2P / npc) / 3.0
                                 * rmincgs ** 3)[:, :, None]
        return rave, dens, vcell

    @staticmethod
    def _disk_rho(w: Workload, autors, rddust, rarr, thetarr):
        """Whitney flared disk on the cell centres (nrg-1, ntg-1):
        rho0 (1-sqrt(R*/w)) w^-a exp(-z^2/2h^2), h = z1 w^b, rho0 from Mdisk."""
        rave = 0.5 * (rarr[:-1] + rarr[1:])
        thave = 0.5 * (thetarr[:-1] + thetarr[1:])
        rad = rave[:, None]
        th = thave[None, :]
        wcyl = rad * np.sin(th)
        zp = rad * np.abs(np.cos(th))
        rmincgs = w.rstar * RSOL
        rmaxd = w.rmaxd_au * autors
        z1 = w.h100_au * autors / (100.0 * autors) ** w.b_exp
        p = w.b_exp - w.a_exp
        const = R2P ** 1.5 * rmincgs ** 2 * (rmincgs * z1)
        rmind = rddust
        rho0 = w.massd * MSOL / const / (
            1.0 / (p + 2.0) * (rmaxd ** (p + 2.0) - rmind ** (p + 2.0))
            - 1.0 / (p + 1.5) * (rmaxd ** (p + 1.5) - rmind ** (p + 1.5)))
        h = z1 * wcyl ** w.b_exp
        with np.errstate(invalid="ignore", divide="ignore"):
            rho_d = rho0 * (1.0 - np.sqrt(1.0 / wcyl)) * wcyl ** (-w.a_exp) * np.exp(-0.5 * (zp / h) ** 2)
        rho_d = np.where((rad > rddust) & (wcyl <= rmaxd) & (wcyl > 1.0), rho_d, 0.0)
        return np.where(rho_d > 1e-300, rho_d, 0.0)

    def _clump_field(self, nr, nt, npc):
        """Seeded hierarchical clump multiplier with mean 1 (fractal_sph.f90 style)."""
        w = self.w
        rng = np.random.default_rng(w.clump_seed)
        field = np.zeros((nr, nt, npc))
        # hierarchical cascade: each level places children around parents
        nlev = 4
        nchild = max(2, int(round(2.0 ** w.clump_dim)))
        pts = rng.random((nchild, 3))
        for _ in range(nlev - 1):
            scale = 0.5 ** (_ + 1)
            kids = pts[:, None, :] + scale * (rng.random((pts.shape[0], nchild, 3)) - 0.5)
            pts = np.mod(kids.reshape(-1, 3), 1.0)
        ix = np.minimum((pts[:, 0] * nr).astype(int), nr - 1)
        iy = np.minimum((pts[:, 1] * nt).astype(int), nt - 1)
        iz = np.minimum((pts[:, 2] * npc).astype(int), npc - 1)
        np.add.at(field, (ix, iy, iz), 1.0)
        field /= field.mean()
        f = w.clump_mass_frac
        return (1.0 - f) + f * field

    # --------------------------------------------------------------- tables
    def _dust(self):
        w = self.w
        lam_um = np.logspace(math.log10(0.1), math.log10(3000.0), w.nlambda)
        s = (np.log10(lam_um) - np.log10(0.1)) / (np.log10(3000.0) - np.log10(0.1))
        kap = w.kappa0 * lam_um ** -1.5
        alb = 0.5 * (1.0 - s)
        gg = 0.6 * (1.0 - s)
        pl = np.full_like(lam_um, 0.5)
        lamdust = 10000.0 * lam_um                     # dust_5.f90:427
        nudust = 12398.0 / lamdust                     # dust_5.f90:428
        kapd = kap.copy()
        kapd[0] = 0.00001 * kapd[0]                    # dust_5.f90:445
        iv = int(np.max(np.nonzero(lam_um <= 0.55)[0]))
        f = (5500.0 - lamdust[iv]) / (lamdust[iv + 1] - lamdust[iv])
        kappav1 = (1.0 - f) * kapd[iv] + f * kapd[iv + 1]
        kapd = kapd / kappav1
        return nudust, kapd, alb, gg, pl, kappav1

    @staticmethod
    def _opac_interp(nu, nudust, tab):
        """opacset interpolation (dust_5.f90:21-60) vectorised over nu."""
        nu = np.asarray(nu, dtype=float)
        n = nudust.size
        out = np.empty_like(nu)
        hi = nu >= nudust[0]
        lo = nu <= nudust[n - 1]
        mid = ~(hi | lo)
        out[hi] = tab[0]
        out[lo] = tab[n - 1]
        if np.any(mid):
            x = nu[mid]
            # nudust decreasing; i0 = last index with x <= nudust(i0)
            i0 = np.searchsorted(-nudust, -x, side="right") - 1
            i0 = np.clip(i0, 0, n - 2)
            i1 = i0 + 1
            ff = (x - nudust[i1]) / (nudust[i0] - nudust[i1])
            out[mid] = (1.0 - ff) * tab[i1] + ff * tab[i0]
        return out

    def _emission_tables(self, nudust, kapd, alb, nT=500, nnu=513):
        tmin, tmax = 0.1, 200000.0
        lTint = np.log(tmin / 11605.0) + np.arange(nT) * math.log(tmax / tmin) / (nT - 1)
        Tint = np.exp(lTint)
        numax = 32.0
        numin = numax / 1024.0
        nuint = numin + np.arange(nnu) * (numax - numin) / (nnu - 1)
        norm = 0.1539897
        gx, gw = np.polynomial.legendre.leggauss(12)
        gx = 0.5 * (gx + 1.0)
        gw = 0.5 * gw
        kapint = np.zeros((nT, nnu))
        kappar = np.zeros(nT)
        kappa_abs = (1.0 - alb) * kapd
        for i in range(nT):
            T = Tint[i]
            nu1_all = nuint * T
            nu0_all = np.concatenate(([0.0], nu1_all[:-1]))
            chi = self._opac_interp(np.concatenate(([0.0], nu1_all)), nudust, kapd)
            kab = self._opac_interp(np.concatenate(([0.0], nu1_all)), nudust, kappa_abs)
            chi0, chi1 = chi[:-1], chi[1:]
            k0, k1 = kab[:-1], kab[1:]
            dnu = nu1_all - nu0_all
            dx = dnu / T
            nu = nu0_all[:, None] + gx[None, :] * dnu[:, None]
            x = nu / T
            with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
                bx = np.where(x > 0, norm * x ** 3 / np.expm1(x), 0.0)
                dbx = np.where(x > 0, -norm * x ** 4 / (4.0 * np.expm1(x) * np.expm1(-x)), 0.0)
            bx = np.nan_to_num(bx)
            dbx = np.nan_to_num(dbx)
            ff = gx[None, :]
            kb = ((1.0 - ff) * k0[:, None] + ff * k1[:, None]) * bx
            cdb = dbx / ((1.0 - ff) * chi0[:, None] + ff * chi1[:, None])
            seg = (kb * gw[None, :]).sum(axis=1)
            segc = (cdb * gw[None, :]).sum(axis=1)
            ok = (nu0_all / T) < 50.0
            seg = np.where(ok, seg, 0.0)
            segc = np.where(ok, segc, 0.0)
            kapint[i] = np.cumsum(dx * seg)
            kappar[i] = 1.0 / np.sum(dx * segc)
        kappap = kapint[:, -1].copy()
        kapint = kapint / kapint[:, -1:]
        kapint[:, -1] = 1.0
        return lTint, Tint, nuint, kapint, kappap, kappar

    def _atmosphere(self, tstar_ev, nhnu=2000):
        lam = np.logspace(math.log10(0.05), math.log10(1000.0), nhnu)   # file order: increasing lambda
        winv = (1.0 / lam)[::-1]                                        # starbarb_2.f90:69-72
        nu = 1.2398 * lam ** -1
        x = nu / tstar_ev
        with np.errstate(over="ignore"):
            f = 0.1539897 * x ** 3 / np.expm1(x)                       # mathsubs.f90:4-22
        f = f[::-1]
        atmosnu = 1.2398 * winv
        hnuint = np.zeros(nhnu)
        hnuint[1:] = np.cumsum(0.5 * (f[1:] + f[:-1]) * (winv[1:] - winv[:-1]))
        hnuint = hnuint / hnuint[-1]
        lognu = np.log10(atmosnu)
        with np.errstate(divide="ignore"):
            loghnu = np.where(hnuint > 0, np.log10(np.maximum(hnuint, 1e-300)), 0.0)
        loghnu[0] = 0.0
        return atmosnu, hnuint, lognu, loghnu

    @staticmethod
    def _accretion_cdf(rarr, rin, rout):
        """Ldint(nrg-1): cumulative disk-accretion luminosity, the table
        initpacc draws the emitting radius from (diskprofile_model11.f90:
        170-227 builds it from its disk structure).  Here the viscous-disk
        profile dL ~ r^-2 (1 - r^-1/2) dr (r in stellar radii) between the
        dust radius and the disk edge.  initpacc takes cell j when
        Ldint(j) <= xi < Ldint(j+1) (locate), so Ldint(j) holds the
        luminosity of the cells before j, normalised to the total."""
        a = np.clip(rarr[:-1], rin, rout)
        b = np.clip(rarr[1:], rin, rout)
        lum = (1.0 / a - 1.0 / b) - (2.0 / 3.0) * (a ** -1.5 - b ** -1.5)
        lum = np.maximum(lum, 0.0)
        cum = np.concatenate([[0.0], np.cumsum(lum[:-1])])
        return cum / cum[-1] if cum[-1] > 0 else cum

    # ---------------------------------------------------------------- build
    def _build(self):
        w = self.w
        (autors, rddust, rmax, rarr, r2arr, thetarr, costarr, sintarr, tan2arr,
         phiarr, aarr, barr) = self._walls()
        rave, dens, vcell = self._densities(autors, rddust, rmax, rarr, thetarr, w.npg)
        nrg, ntg, npg = w.nrg, w.ntg, w.npg
        findopac = np.zeros((nrg, ntg, npg, NDG2), dtype=np.int32)
        for idd in range(NDG2):
            findopac[..., idd] = idd + 1 if idd < 8 else 1       # findopacid_5.f90:97
        tstar = w.tstar_k / 11605.0
        tdust = np.full((nrg, ntg, npg), 0.1 / 11605.0)
        diffus = np.zeros((nrg, ntg, npg), dtype=np.int32)
        diffdir = np.zeros((nrg, ntg, npg), dtype=np.int32)

        nudust, kapd, alb, gg, pl, kappav1 = self._dust()
        nopac = 8
        nl = nudust.size
        lTint, Tint, nuint, kapint1, kappap1, kappar1 = self._emission_tables(nudust, kapd, alb)
        nT, nnu = lTint.size, nuint.size
        rep = lambda a: np.repeat(a[..., None], nopac, axis=-1)
        atmosnu, hnuint, lognu, loghnu = self._atmosphere(tstar)

        numin = 1.2398 / 5000.0                       # setup.f90:36-41
        numax = 1.2398 / 0.01
        nmu = w.nmu
        dmu = 2.0 / nmu
        u = 1.0 - dmu * (np.arange(1, nmu + 1) - 0.5)  # initarr_2_new.f90:22-26
        thete = np.linspace(5.0, 86.0, w.npeel) if w.npeel > 1 else np.array([45.0])
        thete_rad = thete * R2P / 360.0
        phie = np.zeros(w.npeel)
        aperture2 = (w.aperture_au * autors) ** 2 * np.ones(w.nap)

        xmu = np.arange(1, 101) / 100.0               # samptabl.f90:1-23
        prob = 0.5 * (xmu ** 3 + xmu ** 2)
        prob[0] = 0.0

        self.config = dict(
            nrg=nrg, ntg=ntg, npg=npg, nopac=nopac, nlammax=nl, nT=nT, nnu=nnu,
            nhnu=atmosnu.size, nfreq=w.nfreq, nmu=nmu, nph=w.nph, nap=w.nap,
            npeel=w.npeel, nxhst=w.nxhst, output_imcube=1, partial_peeloff=0,
            limb=0, iplanckst=1, idust=1, ilucy=1, iffuv=0, ispot=0, nspot=1,
            rstar=w.rstar, tstar=tstar, tstarave=tstar, tshock=tstar, fspot=0.0,
            accfrac=0.0, accfrac2=0.0, isrf_frac=0.0, rddust=rddust,
            rmaxi=w.rmaxi_au * autors, numin=numin, lnurat=math.log(numax / numin),
            autors=autors,
            ifuv_ori=SIGT * (tstar * 11605.0) ** 4 * 4.0 * PI * (w.rstar * RSOL) ** 2,
        )
        F = lambda a: np.asfortranarray(a).ravel(order="F")
        self.grid = dict(
            rarr=rarr, r2arr=r2arr, thetarr=thetarr, costarr=costarr, sintarr=sintarr,
            tan2arr=tan2arr, phiarr=phiarr, aarr=aarr, barr=barr,
            densarr=F(dens), findopac=F(findopac), diffus=F(diffus), diffdir=F(diffdir),
            tdust=F(tdust), vcell=F(vcell), ravearr=rave,
            Ldint=self._accretion_cdf(rarr, rddust, w.rmaxd_au * autors),
            hdisk=(w.h100_au * autors / (100.0 * autors) ** w.b_exp) * rave ** w.b_exp,
        )
        self.tables = dict(
            nlambda=np.full(nopac, nl, dtype=np.int32),
            nudust=F(rep(nudust)), kappad=F(rep(kapd)), adust=F(rep(alb)),
            gdust=F(rep(gg)), pldust=F(rep(pl)),
            kappav=np.full(nopac, kappav1),
            kapint=F(rep(kapint1)), lTint=lTint, Tint=Tint, nuint=nuint,
            kappap=F(rep(kappap1)), kappar=F(rep(kappar1)),
            atmosnu=atmosnu, hnuint=hnuint, lognu=lognu, loghnu=loghnu,
            aperture2=aperture2, u=u,
            coste_arr=np.cos(thete_rad), sinte_arr=np.sin(thete_rad),
            cospe_arr=np.cos(phie), sinpe_arr=np.sin(phie),
            limb_prob=prob,
        )
        self.ncells = (nrg - 1) * (ntg - 1) * (npg - 1)

    # convenience views (reference shapes)
    def dens4(self):
        w = self.w
        return self.grid["densarr"].reshape((w.nrg, w.ntg, w.npg, NDG2), order="F")


def reference_2d(**over) -> Model:
    """2-D disk+envelope+cavity workload (nr=100, ntheta=99, nphi=1)."""
    return Model(Workload(**over))


def small_2d(**over) -> Model:
    """A reduced grid of the same model for quick oracle comparisons."""
    kw = dict(nrg=31, ntg=21, npg=2, nfreq=20, nmu=4, nph=1, npeel=3, nxhst=21, rim_walls=8)
    kw.update(over)
    return Model(Workload(**kw))


def clumpy_3d(**over) -> Model:
    """3-D clumpy model: nr=200, ntheta=199, nphi=64 cells."""
    kw = dict(nrg=201, ntg=199, npg=65, nph=1, npeel=20, nfreq=20, nxhst=201,
              clump_seed=31944)
    kw.update(over)
    return Model(Workload(**kw))


def warm(m: Model, t1au_k: float = 300.0, q: float = 0.5) -> Model:
    """Give the dust a power-law temperature T = t1au (r/1AU)^-q (cells with
    dust only), a stand-in for a converged Lucy temperature in tests."""
    w = m.w
    autors = m.config["autors"]
    rave = 0.5 * (m.grid["rarr"][:-1] + m.grid["rarr"][1:])
    T = np.full((w.nrg, w.ntg, w.npg), 0.1 / 11605.0)
    tr = np.clip(t1au_k * (rave / autors) ** (-q), 2.0, 1500.0) / 11605.0
    T[:-1, :, :] = tr[:, None, None]
    has = m.dens4().sum(axis=-1) > 0
    T = np.where(has, T, 0.1 / 11605.0)
    m.grid["tdust"] = np.asfortranarray(T).ravel(order="F")
    return m


def _chiR(tables, T, species):
    """chiR (dust_5.f90:112-141): Rosseland table interpolated in log T."""
    lTint = tables["lTint"]
    nT = lTint.size
    kr = tables["kappar"].reshape((nT, -1), order="F")[:, species - 1]
    lT = math.log(T)
    k = int((nT - 1) * (lT - lTint[0]) / (lTint[-1] - lTint[0])) + 1
    k = min(max(k, 1), nT - 1)
    f = (lT - lTint[k - 1]) / (lTint[k] - lTint[k - 1])
    return (1.0 - f) * kr[k - 1] + f * kr[k]


def setdiffus(m: Model, tdave: np.ndarray, iteration: int) -> Model:
    """Flag the optically thick disk interior for the diffusion treatment.

    Restates setdiffus (setdiffus_5.f90:1-132): for every radius inside the
    disk, march from each theta cell toward the pole accumulating the
    Rosseland optical depth; cells whose photon mean free path to tau=1 is
    below h/20 become diffusion cells with diffdir=-2 (upper hemisphere),
    mirrored with diffdir=+2 below the midplane.  kapd is taken at its V-band
    value kappav*R*, the value setup_wave.f90:50 leaves in it.
    """
    w = m.w
    nrg, ntg, npg = w.nrg, w.ntg, w.npg
    dens = m.dens4()
    td = np.asarray(tdave).reshape((nrg, ntg, npg), order="F")
    rarr, thetarr = m.grid["rarr"], m.grid["thetarr"]
    autors = m.config["autors"]
    rmaxd = w.rmaxd_au * autors
    hdisk = m.grid["hdisk"]
    kv = m.tables["kappav"]
    rmincgs = w.rstar * RSOL
    fo = m.grid["findopac"].reshape((nrg, ntg, npg, NDG2), order="F")
    diffus = np.zeros((nrg, ntg, npg), dtype=np.int32)
    diffdir = np.zeros((nrg, ntg, npg), dtype=np.int32)
    thermal = [True, True, True, True, False, False, False, False, True, True]
    if w.massd > 0.0:
        nr0 = 1 if m.config["rddust"] == rarr[0] else 3
        ir = nr0
        rad = rarr[ir - 1]
        while rad < rmaxd and ir <= nrg - 1:
            zmr = hdisk[ir - 1]
            for it in range((ntg - 1) // 2, 1, -1):
                tau = 0.0
                tau1 = 0.0
                itt = it
                while tau < 1.0 and itt > 1:
                    dt = thetarr[itt] - thetarr[itt - 1]
                    tau1 = tau
                    tt = td[ir - 1, itt - 1, 0]
                    if iteration < 2:
                        tt = max(tt, 50.0 / 11605.0)
                    for idd in range(NDG2):
                        if thermal[idd] and dens[ir - 1, itt - 1, 0, idd] > 0.0:
                            sp = int(fo[ir - 1, itt - 1, 0, idd])
                            tau += (kv[sp - 1] * rmincgs) * _chiR(m.tables, tt, sp) * \
                                dens[ir - 1, itt - 1, 0, idd] * dt * rad
                    itt -= 1
                if tau > 1.0:
                    lmfp1 = rad * (thetarr[itt + 1] - thetarr[itt]) / (tau - tau1) * (1.0 - tau1)
                else:
                    lmfp1 = rad * (thetarr[itt + 1] - thetarr[itt])
                lmfp = rad * (thetarr[it] - thetarr[itt + 1]) + lmfp1
                if tau >= 1.0 and lmfp < zmr / 20.0:
                    diffus[ir - 1, it - 1:(ntg - 1) // 2, 0] = 1
                    diffdir[ir - 1, it - 1:(ntg - 1) // 2, 0] = -2
            ir += 1
            rad = rarr[ir - 1]
        for it in range((ntg + 1) // 2, ntg):
            diffus[:nrg - 1, it - 1, 0] = diffus[:nrg - 1, ntg - it - 1, 0]
            diffdir[:nrg - 1, it - 1, 0] = -diffdir[:nrg - 1, ntg - it - 1, 0]
        if npg > 2:
            diffus[:nrg - 1, :ntg - 1, 1:npg - 1] = diffus[:nrg - 1, :ntg - 1, :1]
            diffdir[:nrg - 1, :ntg - 1, 1:npg - 1] = diffdir[:nrg - 1, :ntg - 1, :1]
    # cells without a thermal component cannot diffuse
    has_th = (dens[..., [0, 1, 2, 3, 8, 9]] > 0).any(axis=-1)
    diffus = np.where(has_th, diffus, 0)
    diffdir = np.where(has_th, diffdir, 0)
    m.grid["diffus"] = np.asfortranarray(diffus).ravel(order="F")
    m.grid["diffdir"] = np.asfortranarray(diffdir).ravel(order="F")
    # gridset_5_model13new.f90:1855-1866: tdust of diffusion cells restarts at 0.1 K
    T = np.where(diffus > 0, 0.1 / 11605.0, td)
    T = np.where(dens.sum(axis=-1) > 0, T, 0.1 / 11605.0)
    m.grid["tdust"] = np.asfortranarray(T).ravel(order="F")
    m.config["diffusion"] = True      # gridset reruns setdiffus every iteration (mctherm.par DIFFUSION)
    return m


def with_diffusion(m: Model, iteration: int = 2) -> Model:
    """setdiffus on the model's current temperature."""
    return setdiffus(m, m.grid["tdust"].copy(), iteration)


def with_velocities(m: Model) -> Model:
    """The gas velocity field gridset gives the envelope
    (gridset_5_model13new.f90:1372-1412, 1439-1471): Ulrich infall,
    vfall = sqrt(G (M* + Mdisk) / r) at the cell-centre radius, on the walls
    of theta:
        equator, r > Rc:  vr = -vfall sqrt(2 - Rc/r),  vtheta = 0
        equator, r <= Rc: vr = -vfall,  vtheta = vfall sqrt(1 - r/Rc)
        else:             vr = -vfall sqrt(1 + mu/mu0),
                          vtheta = vfall (mu0 - mu)/sin(theta) sqrt(1 + mu/mu0)
    with mu = |cos(theta)| and mu0 the streamline root (zerod.f90); the
    divergence from the face averages of the upper hemisphere, mirrored
    below.  Cells of the envelope component (id 3) take these values; the
    disk and the cavity stay at rest (this model has no disk wind and no
    expanding outer envelope, so the reference's wind and sonic-point
    branches do not arise).  The pole walls, where the reference's vtheta
    is 0/0, get vtheta = 0."""
    w = m.w
    nrg, ntg, npg = w.nrg, w.ntg, w.npg
    autors = m.config["autors"]
    rarr, thetarr = m.grid["rarr"], m.grid["thetarr"]
    rave = 0.5 * (rarr[:-1] + rarr[1:])
    rc = w.rc_au * autors
    vfall = np.sqrt(GN * (w.massc + w.massd) * MSOL / rave / w.rstar / RSOL)      # [nrg-1]
    vru = np.zeros((nrg, ntg))
    vtu = np.zeros((nrg, ntg))
    sint = np.sin(thetarr)
    cost = np.abs(np.cos(thetarr))
    rx = rave / rc
    for ir in range(nrg - 1):
        mu0 = Model._ulrich_mu0(cost.copy(), np.full(ntg, rx[ir]))
        vr = -vfall[ir] * np.sqrt(1.0 + cost / mu0)
        with np.errstate(invalid="ignore", divide="ignore"):
            vt = np.where(sint > 1e-12, vfall[ir] * (mu0 - cost) / sint * np.sqrt(1.0 + cost / mu0), 0.0)
        ieq = (ntg + 1) // 2 - 1
        if ntg % 2 == 1:
            if rave[ir] > rc:
                vr[ieq] = -vfall[ir] * math.sqrt(2.0 - rc / rave[ir])
                vt[ieq] = 0.0
            else:
                vr[ieq] = -vfall[ir]
                vt[ieq] = vfall[ir] * math.sqrt(1.0 - rave[ir] / rc)
        vru[ir], vtu[ir] = vr, vt
    div = np.zeros((nrg, ntg))
    nu = (ntg - 1) // 2
    for ir in range(nrg - 1):
        rad, rad1, rad2 = rave[ir], rarr[ir + 1], rarr[ir]
        dr = rad1 - rad2
        for it in range(nu):
            t1, t2 = thetarr[it + 1], thetarr[it]
            th = 0.5 * (t1 + t2)
            dt = t1 - t2
            vr1 = 0.5 * (vru[ir + 1, it + 1] + vru[ir + 1, it])
            vr2 = 0.5 * (vru[ir, it + 1] + vru[ir, it])
            vt1 = 0.5 * (vtu[ir + 1, it + 1] + vtu[ir, it + 1])
            vt2 = 0.5 * (vtu[ir + 1, it] + vtu[ir, it])
            div[ir, it] = ((rad1 ** 2 * vr1 - rad2 ** 2 * vr2) / dr / rad ** 2
                           + (math.sin(t1) * vt1 - math.sin(t2) * vt2) / dt / rad / math.sin(th))
        for it in range((ntg + 1) // 2 - 1, ntg - 1):
            div[ir, it] = div[ir, ntg - 2 - it]
    env = m.dens4()[..., 2] > 0.0                   # id 3: envelope
    shape = (nrg, ntg, npg)
    vr3 = np.where(env, np.broadcast_to(vru[:, :, None], shape), 0.0)
    vt3 = np.where(env, np.broadcast_to(vtu[:, :, None], shape), 0.0)
    dv3 = np.where(env, np.broadcast_to(div[:, :, None], shape), 0.0)
    m.grid["vrarr"] = np.asfortranarray(vr3).ravel(order="F")
    m.grid["vthetarr"] = np.asfortranarray(vt3).ravel(order="F")
    m.grid["divvarr"] = np.asfortranarray(dv3).ravel(order="F")
    return m


LUCY_STATE_2D = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "reference_2d_tdave.npy")


def reference_2d_converged(**over) -> Model:
    """The 2-D benchmark model at its converged Lucy temperature: tdave from
    data/reference_2d_tdave.npy (made by data/make_lucy_state.py with the
    FP64 engine) and the diffusion region it implies (setdiffus); the
    power-law stand-in temperature (warm) if the file is absent."""
    m = reference_2d(**over)
    if not over and os.path.exists(LUCY_STATE_2D):
        td = np.load(LUCY_STATE_2D)
        if td.size == m.w.nrg * m.w.ntg * m.w.npg:
            return setdiffus(m, td, 2)
    return with_diffusion(warm(m))


def tdust_from_tdave(m: Model, tdave: np.ndarray) -> np.ndarray:
    """The dust temperature an iteration starts from (gridset_5_model13new.f90:
    1855-1866): tdave, except 0.1 K in diffusion cells and empty cells."""
    w = m.w
    td = np.asarray(tdave, dtype=np.float64).reshape((w.nrg, w.ntg, w.npg), order="F")
    dif = m.grid["diffus"].reshape((w.nrg, w.ntg, w.npg), order="F") > 0
    T = np.where(dif, 0.1 / 11605.0, td)
    T = np.where(m.dens4().sum(axis=-1) > 0, T, 0.1 / 11605.0)
    return np.asfortranarray(T).ravel(order="F")


def with_mueller(m: Model, narr: int = 720, nang: int = 181, s34_frac: float = 0.0) -> Model:
    """Tabulated scattering matrices (stokes6 / tab_mod) for every species
    and wavelength node, generated from the dustmat law (dustmat.f90) with
    each node's g and pmax on `nang` scattering angles (0..180 deg, the
    reference's nar=181 of reatab.f90) and resampled to `narr` uniform
    cosine bins as reatab.f90 does (linearly here), S11 normalised so that
    the sum of S11*dct/2 over the bins is 1.  S11=S22=p1, S12=p2, S33=S44=p3;
    `s34_frac` in [0,1] adds S34 = s34_frac p1 sqrt(1-pmax^2)(1-mu^2)/(1+mu^2),
    which keeps S11^2 >= S12^2+S33^2+S34^2 and makes scattering generate
    circular polarisation.  Returns the model with tables["mueller"] and
    tables["narr"] set (layout mueller(6,narr,nlammax,nopac))."""
    c = m.config
    nl, nop = c["nlammax"], c["nopac"]
    gd = m.tables["gdust"].reshape((nl, nop), order="F")
    pd = m.tables["pldust"].reshape((nl, nop), order="F")
    th = np.linspace(0.0, PI, nang)
    mu_in = np.cos(th)[::-1]                        # ascending
    dct = 2.0 / narr
    mu = -1.0 + (np.arange(1, narr + 1) - 0.5) * dct
    out = np.zeros((nop, nl, narr, 6))
    for sp in range(nop):
        for j in range(nl):
            g, pl = gd[j, sp], pd[j, sp]
            cb2 = mu_in * mu_in
            temp = (g * g + 1.0) - 2.0 * g * mu_in
            p1 = 1.5 * (1.0 - g * g) / (2.0 + g * g) * (1.0 + cb2) / (temp * np.sqrt(temp))
            p2 = -pl * p1 * (1.0 - cb2) / (1.0 + cb2)
            p3 = p1 * 2.0 * mu_in / (1.0 + cb2)
            p4 = s34_frac * p1 * math.sqrt(max(0.0, 1.0 - pl * pl)) * (1.0 - cb2) / (1.0 + cb2)
            cols = [np.interp(mu, mu_in, v) for v in (p1, p2, p1, p3, p4, p3)]
            tot = np.sum(0.5 * cols[0] * dct)
            out[sp, j] = np.stack(cols, axis=-1) / tot
    m.tables["mueller"] = np.ascontiguousarray(out).ravel()
    m.tables["narr"] = int(narr)
    return m


# ----------------------------------------------------------- disk parameters
DISK_PARAMS = ("massd", "b_exp", "h100_au")


def disk_log_derivatives(m: Model, rel_step: float = 1e-4) -> dict:
    """d log(rho_disk) / d(param) on the model's grid, per disk cell
    (nrg-1, ntg-1): for Mdisk and h(100 AU) with respect to the log of the
    parameter, for the flaring index b with respect to b itself.  Central
    differences of the disk law at fixed walls (the law is smooth; the step
    is far below the Monte Carlo noise of any gradient)."""
    import copy
    w = m.w
    autors = 214.94 / w.rstar
    rddust = w.rddust_au * autors
    rarr = m.grid["rarr"]
    thetarr = m.grid["thetarr"]
    base = Model._disk_rho(w, autors, rddust, rarr, thetarr)
    out = {}
    for name in DISK_PARAMS:
        v = getattr(w, name)
        h = rel_step * (abs(v) if name != "b_exp" else 1.0)
        wp, wm = copy.copy(w), copy.copy(w)
        setattr(wp, name, v + h)
        setattr(wm, name, v - h)
        rp = Model._disk_rho(wp, autors, rddust, rarr, thetarr)
        rm = Model._disk_rho(wm, autors, rddust, rarr, thetarr)
        ok = (base > 0) & (rp > 0) & (rm > 0)
        d = np.zeros_like(base)
        d[ok] = (np.log(rp[ok]) - np.log(rm[ok])) / (2.0 * h)
        if name != "b_exp":
            d = d * v                     # d/d log(param)
        out[name] = d
    return out


def with_disk_params(m: Model, **params) -> Model:
    """The model with its disk component recomputed for new disk parameters
    on the same grid, with the same cells owning the disk and the same
    diffusion flags (the fixed structure an adjoint gradient is taken at)."""
    import copy
    mm = copy.deepcopy(m)
    w = copy.copy(m.w)
    for k, v in params.items():
        setattr(w, k, v)
    autors = 214.94 / w.rstar
    rho = Model._disk_rho(w, autors, w.rddust_au * autors, m.grid["rarr"], m.grid["thetarr"])
    dens = mm.grid["densarr"].reshape((w.nrg, w.ntg, w.npg, NDG2), order="F").copy()
    nr, nt, npc = w.nrg - 1, w.ntg - 1, max(w.npg - 1, 1)
    owned = dens[:nr, :nt, :npc, 1] > 0
    dens[:nr, :nt, :npc, 1] = np.where(owned, rho[:, :, None], 0.0)
    mm.grid["densarr"] = np.asfortranarray(dens).ravel(order="F")
    mm.w = w
    return mm


def batch_models(n: int = 64, seed: int = 20240605) -> list:
    """A seeded parameter sweep of uneven models for the batched launch:
    nr 50-200, ntheta 49-199 (odd: the equator is a wall), nphi 1-32 cells;
    Mdisk log-uniform in 1e-4..0.1 Msun, envelope infall rate log-uniform in
    1e-7..1e-5 Msun/yr, cavity opening angle uniform in 5..40 deg; the dust
    law sampled on 60-140 wavelengths (uneven wavelength sets).  No image
    cube (temperature iterations do not peel)."""
    return [batch_model(w) for w in batch_workloads(n, seed)]


def batch_workloads(n: int = 64, seed: int = 20240605) -> list:
    """The parameters of ``batch_models`` without building the models (a
    sharded sweep builds only its own)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nr = int(rng.integers(50, 201))
        nt = int(rng.integers(24, 100)) * 2 + 1
        nph = int(rng.integers(1, 33))
        out.append(Workload(nrg=nr + 1, ntg=nt, npg=nph + 1,
                            massd=float(10.0 ** rng.uniform(-4.0, -1.0)),
                            rate=float(10.0 ** rng.uniform(-7.0, -5.0)),
                            thet1_deg=float(rng.uniform(5.0, 40.0)),
                            nlambda=int(rng.integers(60, 141))))
    return out


def batch_model(w: Workload) -> Model:
    """One sweep model: no image cube."""
    m = Model(w)
    m.config["output_imcube"] = 0
    return m


def isrf_table(nisrf: int = 200, lmin_um: float = 0.0912, lmax_um: float = 1000.0, av: float = 0.0,
               kext=None) -> np.ndarray:
    """The external-illumination sampling table the engine takes
    (mcrt_tables.isrf, Fortran (nisrf, 3): cdf, log10 cdf, log10 nu [eV]),
    built by the steps of isrf_cdf.f90:67-212: nisrf wavelengths log-spaced
    over (lmin, lmax], frequencies ascending, the spectrum per unit
    frequency times exp(-kappa/kappa_V/1.086 * Av), the trapezoid cumulative,
    normalised, and the first row as that routine leaves it (cdf 0, log cdf
    -99, log nu 0).  The spectrum is a synthetic stand-in for the reference's
    tabulated one (not present here): the three diluted blackbodies of the
    stellar interstellar radiation field of Mathis, Mezger & Panagia (1983),
    W = 1e-14, 1e-13, 4e-13 at T = 7500, 4000, 3000 K.  `kext(lam_um)`: the
    extinction curve relative to V for Av > 0."""
    c = 2.99792458e14                                 # um/s
    h_k = 4.799243e-11                                # h/k [K s]
    freq = np.empty(nisrf)
    for i in range(1, nisrf + 1):
        lam = lmin_um * (lmax_um / lmin_um) ** (i / nisrf)
        freq[nisrf - i] = c / lam
    def bnu(nu, T):
        x = h_k * nu / T
        return nu ** 3 / np.expm1(x)
    pdf = sum(W * bnu(freq, T) for W, T in ((1e-14, 7500.0), (1e-13, 4000.0), (4e-13, 3000.0)))
    if av > 0.0:
        pdf = pdf * np.exp(-np.asarray(kext(c / freq)) / 1.086 * av)
    cdf = np.zeros(nisrf)
    for i in range(1, nisrf):
        cdf[i] = cdf[i - 1] + 0.5 * (pdf[i] + pdf[i - 1]) * (freq[i] - freq[i - 1])
    logcdf = np.zeros(nisrf)
    logfreq = np.zeros(nisrf)
    cdf[1:] = cdf[1:] / cdf[-1]
    cdf[0] = 0.0
    logcdf[0] = -99.0
    logfreq[0] = 0.0
    logcdf[1:] = np.log10(cdf[1:])
    logfreq[1:] = np.log10(freq[1:] * 1.2398 / c)
    return np.concatenate([cdf, logcdf, logfreq])


def with_isrf(m: Model, frac: float = 0.2, **kw) -> Model:
    """External-illumination packets (isrf_frac): a fraction `frac` of every
    iteration's packets enters from the outer sphere with the ISRF spectrum
    of ``isrf_table``."""
    t = isrf_table(**kw)
    m.tables["isrf"] = t
    m.tables["nisrf"] = t.size // 3
    m.config["isrf_frac"] = frac
    return m


def filter_table(bands_um=(3.6, 24.0, 70.0), rel_width: float = 0.25, npts: int = 60, nwfiltmax: int = 64):
    """Filter curves in the layout filt_nu.f90 leaves in filt_mod: per
    filter, frequencies in Hz (2.9979e14 / lambda[um]) ascending over its
    points, responses normalised by their trapezoidal integral over
    frequency (filt_nu.f90:50-103), padded to nwfiltmax points; nwfilt
    counts the points plus the file's header line, as the reference does.
    The reference reads its 49 curves (2MASS, IRAC, MIPS, ...) from files that
    are not present; here band b is a Gaussian in log wavelength centred on
    bands_um[b] with relative width rel_width, sampled out to 2.5 widths.
    Returns (nwfilt, filtwave, filtphi), the last two Fortran-ordered
    (nwfiltmax, nfilt)."""
    nf = len(bands_um)
    if npts > nwfiltmax:
        raise ValueError("npts must fit in nwfiltmax")
    nwfilt = np.full(nf, npts + 1, np.int32)
    fw = np.zeros((nwfiltmax, nf))
    fp = np.zeros((nwfiltmax, nf))
    for b, lam0 in enumerate(bands_um):
        x = np.linspace(-2.5, 2.5, npts)
        lam = lam0 * np.exp(x * rel_width)[::-1]             # decreasing wavelength: ascending frequency
        f = 2.9979e14 / lam
        phi = np.exp(-0.5 * ((np.log(lam / lam0)) / rel_width) ** 2)
        fint = np.sum(0.5 * (phi[1:] + phi[:-1]) * (f[1:] - f[:-1]))
        fw[:npts, b] = f
        fp[:npts, b] = phi / fint
        fw[npts:, b] = f[-1]
    F = lambda a: np.asfortranarray(a).ravel(order="F")
    return nwfilt, F(fw), F(fp)


def with_filters(m: Model, **kw) -> Model:
    """Filter-band images (output_imfilt): the curves of ``filter_table``."""
    nwfilt, fw, fp = filter_table(**kw)
    m.tables["nwfilt"] = nwfilt
    m.tables["filtwave"] = fw
    m.tables["filtphi"] = fp
    m.config["output_imfilt"] = 1
    m.config["nfilt"] = int(nwfilt.size)
    m.config["nwfiltmax"] = int(fw.size // nwfilt.size)
    return m


def nested_levels(l_max: float, l_min: float, factor: int):
    """Half sizes of the nested images, ascending, as find_levels
    (type_nested_image.f90:62-73) computes them in single precision:
    n = ceiling(log10(l_max/l_min) / log10(factor)) + 1 and
    levels(n+1-l) = l_max / factor**(l-1)."""
    f32 = np.float32
    lmax, lmin, fac = f32(l_max), f32(l_min), f32(factor)
    n = int(math.ceil(float(np.log10(lmax / lmin) / np.log10(fac)))) + 1
    lev = np.zeros(n, np.float32)
    for l in range(1, n + 1):
        lev[n - l] = lmax / fac ** f32(l - 1)
    return lev


def with_nested_images(m: Model, dim: int = 64, rmax_au: float | None = None, rmin: float = 50.0,
                       factor: int = 4) -> Model:
    """Nested multi-wavelength images (output_imsparse): the setup of
    initarr_2_new.f90:170-190 -- half sizes from rmax_au [AU] (default: the
    image half size) down to rmin [R*], nfreq bins in log10(frequency [Hz])
    over the SED range, both computed in single precision as there."""
    if dim % factor or (dim // 2) % 2:
        raise ValueError("dim must be a multiple of factor and dim/2 even (nested_image_setup)")
    c = m.config
    autors = c["autors"]
    rmax = (m.w.rmaxi_au if rmax_au is None else rmax_au)
    f32 = np.float32
    numin = f32(c["numin"])
    numax = f32(c["numin"] * math.exp(c["lnurat"]))
    c.update(output_imsparse=1, sparse_dim=dim, sparse_nnu=c["nfreq"],
             sparse_lognu_min=float(np.log10(numin * f32(2.9979e14) / f32(1.2398))),
             sparse_lognu_max=float(np.log10(numax * f32(2.9979e14) / f32(1.2398))))
    lev = nested_levels(f32(rmax) * f32(autors), rmin, factor)
    c["sparse_nlev"] = int(lev.size)
    m.tables["sparse_levels"] = lev
    return m


def draine_table(nemit: int = 18, ndraine: int = 1000, lmin_um: float = 1.0, lmax_um: float = 1000.0) -> np.ndarray:
    """Small-grain (VSG/PAH) emission spectra in the layout draine_cdf.f90
    leaves in draine_mod: cdf_d(nemit,ndraine), logcdf_d(nemit,ndraine) and
    logfreq_d(ndraine), concatenated (Fortran order), frequencies ascending
    in eV.  The reference reads Draine's emissivities at 18 intensity ratios
    (uratio_arr 0.5 ... 1e7) from files that are not present; here row j is
    a synthetic spectrum with the aromatic bands (3.3, 6.2, 7.7, 8.6, 11.3,
    12.7, 17 um, Lorentzian profiles) over a modified-blackbody continuum
    whose temperature rises with the intensity ratio (T = 40 K U^(1/6)), the
    continuum's share growing with U.  The table itself follows
    draine_cdf.f90 step for step: the wavelength grid reversed into
    ascending frequency, trapezoidal cumulative sums in frequency, the rows
    normalised, cdf 0 / log cdf -10 / log freq 0 in the first column."""
    uratio = np.array([0.5, 1.0, 2.0, 5.0, 10.0, 20.0, 30.0, 1e2, 3e2, 1e3, 3e3, 1e4, 3e4, 1e5, 3e5, 1e6, 3e6, 1e7])
    uratio = uratio[:nemit] if nemit <= uratio.size else np.logspace(-0.3, 7.0, nemit)
    lam = np.logspace(math.log10(lmin_um), math.log10(lmax_um), ndraine)       # file order: increasing lambda
    bands = [(3.3, 0.04, 0.3), (6.2, 0.15, 1.0), (7.7, 0.4, 2.0), (8.6, 0.3, 0.8), (11.3, 0.25, 1.5),
             (12.7, 0.3, 0.6), (17.0, 1.0, 0.4)]
    pdf = np.zeros((nemit, ndraine))
    for j, U in enumerate(uratio):
        T = 40.0 * U ** (1.0 / 6.0)
        x = 14387.77 / (lam * T)
        with np.errstate(over="ignore"):
            cont = lam ** -5 / np.expm1(np.minimum(x, 700.0)) * lam ** -1.5
        cont = cont / cont.max()
        aro = sum(a / (1.0 + ((lam - l0) / w) ** 2) for l0, w, a in bands)
        mix = 0.2 + 0.7 * (math.log10(U) + 0.3) / 7.3
        pdf[j] = (1.0 - mix) * aro / aro.max() + mix * cont
    freq = (1.2398 / lam)[::-1]                                  # draine_cdf.f90: freq_d(ndraine-i+1)
    pdf_d = pdf[:, ::-1]
    cdf = np.zeros((nemit, ndraine))
    cdf[:, 1:] = np.cumsum(0.5 * (pdf_d[:, 1:] + pdf_d[:, :-1]) * (freq[1:] - freq[:-1])[None, :], axis=1)
    cdf[:, 1:] = cdf[:, 1:] / cdf[:, -1:]
    cdf[:, 0] = 0.0
    logcdf = np.empty_like(cdf)
    logcdf[:, 0] = -10.0
    logcdf[:, 1:] = np.log10(cdf[:, 1:])
    logfreq = np.empty(ndraine)
    logfreq[0] = 0.0
    logfreq[1:] = np.log10(freq[1:])
    F = lambda a: np.asfortranarray(a).ravel(order="F")
    return np.concatenate([F(cdf), F(logcdf), logfreq])


def with_small_grains(m: Model, fsg: float = 0.2, sg_cavity: bool = True, **kw) -> Model:
    """Small grains (VSG/PAH, component ids 5-8, grid_mod_5.f90:20): a
    fraction `fsg` of the disk's and the envelope's dust mass moves to their
    small-grain components (ids 6 and 7), and with `sg_cavity` the cavity's
    dust becomes small grains only (id 8).  The reference's select_dust
    (select_dust_2.f90:20-33) picks the one thermal component of a cell
    whenever there is exactly one, so small grains absorb and re-emit (from
    the Draine spectra, ``draine_table``) only in cells without thermal dust,
    here the cavity.  Species 5-8 use the dust law of the others."""
    w = m.w
    d = m.dens4().copy()
    d[..., 5] = fsg * d[..., 1]
    d[..., 1] = (1.0 - fsg) * d[..., 1]
    d[..., 6] = fsg * d[..., 2]
    d[..., 2] = (1.0 - fsg) * d[..., 2]
    if sg_cavity:
        d[..., 7] = d[..., 3]
        d[..., 3] = 0.0
    m.grid["densarr"] = np.asfortranarray(d).ravel(order="F")
    t = draine_table(**kw)
    m.tables["draine"] = t
    nemit = kw.get("nemit", 18)
    m.tables["nemit"] = nemit
    m.tables["ndraine"] = t.size // (2 * nemit + 1)
    return m
