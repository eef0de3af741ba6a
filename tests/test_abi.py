"""The C-ABI library loads on a host without a GPU and exports every entry
point include/mcrt_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mcrt_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\s*\*)\s*\*?\s*(mcrt_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("mcrt_create", "mcrt_upload_grid", "mcrt_upload_tables", "mcrt_run_iteration",
                 "mcrt_download_tallies", "mcrt_update_temperature", "mcrt_last_error", "mcrt_destroy"):
        assert must in names


def test_library_exports_all_symbols():
    from src3_mpi_cfitsio_b200 import engine
    lib = engine.load_library()
    for name in declared():
        assert hasattr(lib, name), name
    assert lib.mcrt_version().decode().startswith("mcrt-b200")


def test_struct_sizes_match_header():
    # mirrored ctypes layouts: 24 int32 + 23 double + 8 int32 + 2 float config, pointer-only structs
    from src3_mpi_cfitsio_b200 import abi
    assert ctypes.sizeof(abi.Config) == 24 * 4 + 23 * 8 + 8 * 4 + 2 * 4
    assert ctypes.sizeof(abi.Grid) == 22 * 8
    assert ctypes.sizeof(abi.Tables) == 31 * 8 + 6 * 4
    assert ctypes.sizeof(abi.Tallies) == (4 + 2 + 10 + 9 + 4 + 2 + 8 + 4) * 8
    assert ctypes.sizeof(abi.PacketLog) == 8 + 12 * 4 + 10 * 8


def test_struct_layouts_match_the_c_compiler():
    """The ctypes mirrors have the sizes and member offsets the C compiler
    gives the header's structs."""
    import os
    import shutil
    import subprocess
    import tempfile
    from src3_mpi_cfitsio_b200 import abi
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    structs = {"mcrt_config": abi.Config, "mcrt_grid": abi.Grid, "mcrt_tables": abi.Tables,
               "mcrt_tallies": abi.Tallies, "mcrt_packet_log": abi.PacketLog,
               "mcrt_device_tallies": abi.DeviceTallies, "mcrt_density_params": abi.DensityParams}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mcrt_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write("\n".join(lines))
        subprocess.run([cc, "-I", inc, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_setemiss_rejects_bad_tables_without_a_gpu():
    """mcrt_setemiss checks its inputs before any CUDA call: a wavelength
    column whose nu does not decrease is refused with a message."""
    from src3_mpi_cfitsio_b200.engine import MCRTError, setemiss
    nud = np.array([1.0, 2.0, 0.5])
    with pytest.raises(MCRTError, match="decrease"):
        setemiss(nud, np.ones(3), np.zeros(3), [3])
    with pytest.raises(MCRTError, match="nT"):
        setemiss(np.array([2.0, 1.0]), np.ones(2), np.zeros(2), [2], nT=10)


def test_model_density_and_batch_refuse_bad_input_without_a_gpu():
    """mcrt_model_density checks its walls and parameters, and
    mcrt_batch_create its context list, before any CUDA call."""
    import ctypes as C
    from src3_mpi_cfitsio_b200 import abi, model
    from src3_mpi_cfitsio_b200.engine import density_params, load_library
    lib = load_library()
    m = model.small_2d()
    p = density_params(m.w)
    r = np.ascontiguousarray(m.grid["rarr"][::-1])           # decreasing walls
    t = np.ascontiguousarray(m.grid["thetarr"])
    out = np.zeros(m.w.nrg * m.w.ntg * m.w.npg * 10)
    vc = np.zeros(m.w.nrg * m.w.ntg * m.w.npg)
    D = C.POINTER(C.c_double)
    rc = lib.mcrt_model_density(0, C.byref(p), m.w.nrg, m.w.ntg, m.w.npg, r.ctypes.data_as(D), t.ctypes.data_as(D),
                                None, out.ctypes.data_as(D), vc.ctypes.data_as(D), None)
    assert rc == 1 and b"rarr" in lib.mcrt_last_error(None)
    p.thet1_deg = 95.0
    rc = lib.mcrt_model_density(0, C.byref(p), m.w.nrg, m.w.ntg, m.w.npg, t.ctypes.data_as(D), t.ctypes.data_as(D),
                                None, out.ctypes.data_as(D), vc.ctypes.data_as(D), None)
    assert rc == 1 and b"parameters" in lib.mcrt_last_error(None)
    h = C.c_void_p()
    assert lib.mcrt_batch_create(None, 2, C.byref(h)) == 1 and not h.value
    arr = (C.c_void_p * 2)(None, None)
    assert lib.mcrt_batch_create(arr, 2, C.byref(h)) == 1 and not h.value


def _bad(m, key, index, value):
    import copy
    b = copy.deepcopy(m)
    a = np.array(b.grid[key], dtype=np.float64, copy=True)
    a[index] = value
    b.grid[key] = a
    return b


def test_grid_check_accepts_the_models():
    """mcrt_check_grid runs on the host alone (no device is touched)."""
    from src3_mpi_cfitsio_b200 import engine, model
    for m in (model.small_2d(), model.reference_2d_converged()):
        rc, msg = engine.check_grid(m)
        assert rc == 0 and msg == ""


@pytest.mark.parametrize("key,index,value,word", [("densarr", 5000, float("nan"), "densarr"),
                                                  ("densarr", 7, -1e-20, "densarr"),
                                                  ("tdust", 100, float("inf"), "tdust"),
                                                  ("vcell", None, 0.0, "vcell"),
                                                  ("rarr", 3, 0.5, "rarr"),
                                                  ("costarr", 4, float("nan"), "theta")])
def test_grid_check_refuses_bad_values(key, index, value, word):
    """A non-finite or negative density or temperature, a dust cell without
    volume and non-increasing walls are refused with MCRT_ERR_ARG (1) and the
    entry named, before any CUDA call; the driver's data is not touched."""
    from src3_mpi_cfitsio_b200 import engine, model
    m = model.small_2d()
    if index is None:      # the first cell that holds dust
        index = int(np.flatnonzero(m.dens4().reshape(-1, m.dens4().shape[-1], order="F").sum(axis=1) > 0)[0])
    rc, msg = engine.check_grid(_bad(m, key, index, value))
    assert rc == 1 and word in msg, msg
