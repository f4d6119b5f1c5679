"""The C-ABI library loads and exports every entry point that
include/g1sim_b200.h declares (no GPU needed: nothing is called)."""
import ctypes
import os
import re

from g1sim_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "g1sim_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|char|size_t|float|double|unsigned)\s*\*?\s*(\w+)\s*\(",
                       txt, re.M)
    return sorted(set(names))


def test_header_declares_reference_names():
    names = declared_functions()
    for ref in ("g1_cuda_step", "g1_cuda_reset_done"):
        assert ref in names
    assert len(names) >= 10, names
    # every function prototype in the header is seen by the scan above
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "g1sim_b200.h")).read(), flags=re.S)
    protos = re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;{]*\)\s*;", txt, re.M)
    assert set(protos) <= set(names), sorted(set(protos) - set(names))


def test_library_exports_every_declared_symbol():
    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_build_targets_sm100a_only():
    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "compute_90" not in flags and "sm_80" not in flags
