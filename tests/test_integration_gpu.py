"""The reference's own callers with libhme behind their seams.

oracle/_ref/seams/seam_check (built by integration/Makefile from the reference's
headers and CPU engine, integration/HmeSeams.cpp and libhme) installs hme as
the ring2k device LU table (ring2k::device::set_ops) and as the device RREF
hook (elim::set_device_rref_hook), then runs the reference's
ring2k::echelon_blocked / smith / howell (u32 and u64 rungs; resident and
tiled windows; serial and threaded routes; the reference's own verify twin)
and elim::rref / column_rank_profile / inverse / solve_multi_rhs, and checks
every result entry for entry against the same calls on the host route."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "seams", "seam_check")

pytestmark = pytest.mark.gpu


def test_reference_callers_through_hme_seams():
    if not os.path.exists(EXE):
        pytest.skip("the seam check is built only where the reference sources are present")
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=900)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-6000:]
    assert "0 failed" in out


TAPE = os.path.join(ROOT, "oracle", "_ref", "seams", "tape_check")


def test_reference_tape_on_the_hme_device_layer():
    """The reference's tape -- Recorder, compile, Executor and DeviceBackend compiled
    unchanged from its sources -- linked against integration/HmeEngineCuda.cpp (the
    reference's engine::cuda layer over libhme) in place of the reference's
    libEngineCuda: u32 and u64 programs (GEMM, Schur update, AXPY, SCAL, TRANSPOSE,
    row-list GATHER; row- and column-major operands) on the device, the second run
    from a captured CUDA graph, equal entry for entry to the CPU run; one program
    under the executor's own device verify twin."""
    if not os.path.exists(TAPE):
        pytest.skip("the tape check is built only where the reference sources are present")
    r = subprocess.run([TAPE], capture_output=True, text=True, timeout=900)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-6000:]
    assert "0 failed" in out
