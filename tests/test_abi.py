"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
entry point declared in include/fastice_b200.h (no compute calls here)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fastice_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fi_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "fi_model_create" in names and "fi_model_advance" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(fi):
    for flavor in ("fast", "strict"):
        lib = fi.load_library(flavor)
        missing = [n for n in declared_functions() if not hasattr(lib, n)]
        assert not missing, (flavor, missing)


def test_python_binding_covers_header(fi):
    bound = {name for name, _, _ in fi._lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_build_targets_sm100a():
    mk = open(os.path.join(ROOT, "fastice.jl_b200", "Makefile")).read()
    assert "arch=compute_100a,code=sm_100a" in mk


def test_create_without_gpu_fails_cleanly(fi):
    import torch
    if torch.cuda.is_available():
        return
    g = fi.UniformGrid(origin=(0, 0), extent=(1, 1), dims=(8, 8))
    try:
        fi.IsothermalFullStokesModel(grid=g, boundary_conditions=dict(x=(fi.SBC(0, 0), fi.SBC(0, 0)),
                                                                      y=(fi.SBC(0, 0), fi.SBC(0, 0))),
                                     gravity=dict(x=0.0, y=0.0), rheology=fi.LinearViscousRheology(1.0),
                                     solver_params=fi.pt_params(g))
    except fi.FastIceError as e:
        assert e.status == 5
    else:
        raise AssertionError("model creation must fail without a CUDA device")


def test_abi_version(fi):
    assert fi.load_library().fi_abi_version() == 1
