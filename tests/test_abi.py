"""The C-ABI library loads and exports every entry point include/dsgpu.h declares (no GPU needed)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "dsgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dsg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "dsg_init" in names and "dsg_gate_run" in names
    assert len(names) >= 6


def test_library_exports_every_declared_symbol():
    import dsgpu
    lib = ctypes.CDLL(dsgpu.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_no_gpu_reports_error_not_exit():
    """Without a usable device the library returns an error code instead of exiting."""
    import torch
    if torch.cuda.is_available():
        return
    import dsgpu
    rc = dsgpu.lib.dsg_init(ctypes.c_int(0), ctypes.c_float(0.35))
    assert rc < 0
    assert dsgpu.lib.dsg_last_error()
