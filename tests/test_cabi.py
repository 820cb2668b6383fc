"""The C ABI library loads on a machine without a GPU, exports every entry
point include/*.h declares, and fails cleanly (no exit, no crash) where a
GPU is needed."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import REPO

import d3q19_b200 as d3


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\**\s*(d3q19_[a-z_0-9]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "d3q19_create" in names and "d3q19_step" in names and len(names) >= 20


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    lib = C.CDLL(d3.CUDA_LIB)
    assert getattr(lib, name) is not None


def test_struct_sizes_match_reference_layout():
    assert C.sizeof(d3.IntParams) == 332 and C.sizeof(d3.FlpParams) == 176


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_create_without_gpu_returns_enodev():
    cfg = d3.parse_config("total_lattice_size 8 8 8\n")
    hs = d3.HostState(cfg, data_dir=".")
    with pytest.raises(d3.D3Q19Error, match="ENODEV"):
        d3.Simulation(hs.cfg.ip, hs.cfg.fp, hs.options)


def test_invalid_parameters_rejected_before_device_use():
    lib = d3.cuda_lib()
    cfg = d3.parse_config("total_lattice_size 8 8 8\nboundary_conditions_xyz 1 1 0\n")
    h = C.c_void_p()
    rc = lib.d3q19_create(C.byref(cfg.ip), C.byref(cfg.fp), C.byref(d3.Options()), C.byref(h))
    assert rc == -1 and b"velocity boundaries" in lib.d3q19_last_error(None)
    cfg = d3.parse_config("total_lattice_size 8 8 8\nlattice_buffer_size 2 2 2\n")
    assert lib.d3q19_create(C.byref(cfg.ip), C.byref(cfg.fp), C.byref(d3.Options()), C.byref(h)) == -1


def test_tuning_table_round_trip_without_gpu():
    """The grid autotuner's table (d3q19_tune_import/export/clear) is host
    state: lines in the export format come back unchanged; a malformed line
    adds nothing."""
    d3.tune_clear()
    line = "NVIDIA B200\t148\t1\t0\t11\t3\t2\t412.5\n"
    d3.tune_import(line)
    assert d3.tune_export() == line
    # A later line of the same class replaces the entry.
    d3.tune_import(line.replace("\t3\t2\t412.5", "\t4\t1\t400"))
    assert d3.tune_export() == line.replace("\t3\t2\t412.5", "\t4\t1\t400")
    for bad in ("NVIDIA B200\t148\t1\t0\t11\t3\t2\n",          # a field missing
                "NVIDIA B200\t148\t3\t0\t11\t3\t2\t1.0\n",      # storage out of range
                "NVIDIA B200\t148\t1\t0\t11\t3\t0\t1.0\n",      # no particle CTAs
                "NVIDIA B200\t148\t1\t0\t11\t3\t2\tfast\n",     # not a number
                "\t148\t1\t0\t11\t3\t2\t1.0\n"):                # no device name
        with pytest.raises(d3.D3Q19Error, match="EINVAL"):
            d3.tune_import("H100\t132\t0\t0\t9\t2\t1\t5.0\n" + bad)
    assert "H100" not in d3.tune_export()
    d3.tune_clear()
    assert d3.tune_export() == ""


def test_tuning_cache_file(tmp_path, monkeypatch):
    """D3Q19_TUNE_CACHE: the table is written to the file and read back."""
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("D3Q19_TUNE_CACHE", str(path))
    d3.tune_clear()
    d3.tune_import("NVIDIA B200\t148\t0\t1\t12\t4\t2\t300\n")
    d3._tune_cache_save()
    d3.tune_clear()
    monkeypatch.setattr(d3, "_TUNE_LOADED", False)
    d3._tune_cache_load()
    assert d3.tune_export() == path.read_text() == "NVIDIA B200\t148\t0\t1\t12\t4\t2\t300\n"
    d3.tune_clear()
