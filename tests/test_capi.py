"""CPU tests of the C ABI: libhme builds, loads, and exports (and the ctypes
layer binds) every entry point declared in include/hme.h.  No GPU compute."""
import os
import re
import subprocess

import numpy as np

import hacs_b200
from hacs_b200 import _lib, gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "hme.h")).read()
    return sorted(set(re.findall(r"HME_API\s+[\w\s\*]+?\b(hme_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "hme_gemm_u32" in names and "hme_gemm_u32_dev" in names and len(names) >= 10


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        hacs_b200.build()
    out = subprocess.check_output(["nm", "-D", "--defined-only", _lib.LIB_PATH], text=True)
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in declared() if n not in exported]
    assert not missing, f"declared in include/hme.h but not exported: {missing}"


def test_ctypes_binds_every_declared_symbol():
    L = _lib.lib()
    for n in declared():
        assert n in _lib.PROTOTYPES, f"{n} has no ctypes prototype"
        getattr(L, n)


def test_host_checksum_matches_reference_formula():
    M = gen.engine_matrix(17, 23, 65521, 1)
    import oracle as O

    assert gen.fnv_matrix(M) == O.fnv_matrix(M)


def test_context_creation_without_a_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        return
    try:
        hacs_b200.Engine(0)
    except hacs_b200.HmeError as e:
        assert e.code in (_lib.HME_ECUDA, _lib.HME_EUNSUPPORTED, _lib.HME_EINVAL)
    else:
        raise AssertionError("a context was created without a device")
