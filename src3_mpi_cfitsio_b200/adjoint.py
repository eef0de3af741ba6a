"""Gradients of peeled SEDs and images (config: adjoint on the 2-D model).

``Engine.adjoint`` (C ABI ``mcrt_adjoint``) returns dL/dlog(rho) per cell
and density component for an objective L that weights the peeled SED ``ti``
and the monochromatic image cube ``image_m_i``.  This module builds such
weights and carries the per-cell gradient to parameters of the density law
by the chain rule:

* ``sed_image_weights``: L = peeled flux summed over all SED bins plus the
  image flux at chosen wavelengths (e.g. 3.6, 24 and 70 um), each weighted
  by a caller-chosen factor;
* ``parameter_gradient``: dL/dlog(Mdisk), dL/db (flaring index) and
  dL/dlog(h(100 AU)) from the disk component's per-cell gradient and the
  disk law's log-derivatives on the fixed grid (``model.disk_log_derivatives``);
* ``finite_difference``: the same derivatives by central differences of the
  objective with common random numbers, the check the gradients are held
  against.
"""
from __future__ import annotations

import numpy as np

from . import model as mdl

DISK_ID = 2            # density component of the disk grains


def freq_bin(m, lam_um: float) -> int:
    """1-based SED frequency bin of a wavelength (propagate_5_fuv.f90's
    inub = nfreq log(nu/numin)/lnurat + 1 with nu = 1.2398/lambda)."""
    c = m.config
    nu = 1.2398 / lam_um
    ib = int(c["nfreq"] * np.log(nu / c["numin"]) / c["lnurat"]) + 1
    return min(max(ib, 1), c["nfreq"])


def sed_image_weights(m, image_um=(3.6, 24.0, 70.0), sed_weight: float = 1.0, image_weight: float = 1.0):
    """(lam_psed, lam_img): the total peeled flux (all SED bins, total
    component, every inclination and aperture) plus the image flux at the
    frequency bins of `image_um` (every pixel and inclination)."""
    c = m.config
    lam = np.zeros((c["nfreq"], c["npeel"], c["nap"], 8))
    lam[:, :, :, 0] = sed_weight
    img = np.zeros((c["npeel"], c["nxhst"], c["nxhst"], c["nfreq"]))
    for lu in image_um:
        img[:, :, :, freq_bin(m, lu) - 1] = image_weight
    return lam.ravel(order="F"), img.ravel(order="F")


def parameter_gradient(m, grad: np.ndarray, dlog: np.ndarray | None = None) -> dict:
    """Chain rule from dL/dlog(rho) (engine layout [ncell*10], Fortran
    (nrg,ntg,npg,10)) to the disk parameters of ``model.DISK_PARAMS``:
    dL/dlog(Mdisk), dL/db, dL/dlog(h100).  `dlog`: the disk law's
    log-derivatives, Fortran (nrg-1, ntg-1, 3), e.g. the analytic ones of
    ``engine.model_density``; default: central differences of the host law."""
    w = m.w
    G = grad.reshape((w.nrg, w.ntg, w.npg, 10), order="F")[:-1, :-1, :max(w.npg - 1, 1), DISK_ID - 1]
    dens = m.grid["densarr"].reshape((w.nrg, w.ntg, w.npg, 10), order="F")[:-1, :-1, :max(w.npg - 1, 1), DISK_ID - 1]
    if dlog is None:
        ders = mdl.disk_log_derivatives(m)
    else:
        D = np.asarray(dlog).reshape((w.nrg - 1, w.ntg - 1, 3), order="F")
        ders = {name: D[:, :, k] for k, name in enumerate(mdl.DISK_PARAMS)}
    out = {}
    for name, d in ders.items():
        out[name] = float(np.sum(np.where(dens > 0, G * d[:, :, None], 0.0)))
    return out


def finite_difference(run_objective, m, rel_step: float = 1e-3) -> dict:
    """Central differences of the objective in the disk parameters, in the
    variables of ``parameter_gradient`` (log Mdisk, b, log h100), with the
    grid, disk cells and diffusion flags held fixed; `run_objective(model)`
    must use common random numbers (the same seeds) for every call."""
    out = {}
    w = m.w
    for name in mdl.DISK_PARAMS:
        v = getattr(w, name)
        if name == "b_exp":
            h = rel_step
            lp = run_objective(mdl.with_disk_params(m, **{name: v + h}))
            lm = run_objective(mdl.with_disk_params(m, **{name: v - h}))
            out[name] = (lp - lm) / (2.0 * h)
        else:
            lp = run_objective(mdl.with_disk_params(m, **{name: v * np.exp(rel_step)}))
            lm = run_objective(mdl.with_disk_params(m, **{name: v * np.exp(-rel_step)}))
            out[name] = (lp - lm) / (2.0 * rel_step)
    return out
