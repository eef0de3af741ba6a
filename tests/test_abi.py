"""The C-ABI library loads on a host without a GPU and exports every entry
point include/mcrt_b200.h declares (no compute calls here)."""
import ctypes
import os
import re

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
    # mirrored ctypes layouts: 24 int32 + 23 double config, pointer-only structs
    from src3_mpi_cfitsio_b200 import abi
    assert ctypes.sizeof(abi.Config) == 24 * 4 + 23 * 8
    assert ctypes.sizeof(abi.Grid) == 18 * 8
    assert ctypes.sizeof(abi.Tables) == 24 * 8
    assert ctypes.sizeof(abi.Tallies) == (4 + 2 + 10 + 9 + 4 + 2) * 8
    assert ctypes.sizeof(abi.PacketLog) == 8 + 12 * 4 + 10 * 8
