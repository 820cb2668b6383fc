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
