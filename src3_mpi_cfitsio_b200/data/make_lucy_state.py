"""Generate reference_2d_tdave.npy: the converged Lucy temperature of the 2-D
benchmark model (disk + Ulrich envelope + cavity, model.reference_2d).

Run on a machine with a GPU, from the repository root:
    python src3_mpi_cfitsio_b200/data/make_lucy_state.py [iterations] [packets]

Starting from the power-law stand-in temperature (model.warm) with the
diffusion region it implies, the FP64 engine runs `iterations` Lucy
iterations of `packets` packets (the reference's loop: `disk` then `tfinal`,
newtts.f90:215-256), re-deriving the diffusion region from each new
temperature (setdiffus, newdisktherm_5_fuv.f90:89).  The last tdave is saved
as float64 in Fortran order (nrg x ntg x npg walls).  The benchmark's GPU arm
and both CPU arms start from this state, so they time the same workload.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main(iterations: int = 12, packets: int = 100_000_000) -> str:
    from src3_mpi_cfitsio_b200 import model
    from src3_mpi_cfitsio_b200.engine import Engine
    m = model.with_diffusion(model.warm(model.reference_2d()))
    td = m.grid["tdust"].copy()
    for it in range(1, iterations + 1):
        eng = Engine(m, device=0, precision="fp64")
        eng.set_schedule("wave")
        eng.tdave = td.copy()
        eng.reset_tallies()
        eng.run(packets, iteration=it, ipeel=0)
        td, conv, sig = eng.update_temperature(packets, it)
        eng.close()
        m = model.setdiffus(m, td, it + 1)
        print(f"iteration {it}: converge={conv} sigma={sig}", flush=True)
    out = os.path.join(HERE, "reference_2d_tdave.npy")
    np.save(out, np.asarray(td, dtype=np.float64))
    return out


if __name__ == "__main__":
    a = [int(x) for x in sys.argv[1:]]
    print(main(*a))
