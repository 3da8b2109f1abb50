"""The allocation-free GEMM entry point, hme_gemm_u32_dev_noalloc.

It exists for callers that cannot allocate device memory when they need a
product (a plugin whose host runtime owns the whole device budget, or a
latency-critical path where cudaMalloc / cudaFree would synchronise the
device): its limb planes live in a fixed 32 MiB scratch array inside the
library.  These tests call it through the C ABI and require its output to equal,
bit for bit (the tolerance of every integer test here is zero), that of the
regular entry point hme_gemm_u32_dev on the same inputs, on two calls in a row
(the second call reuses the scratch the first one left behind).  This file is
named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from hacs_b200 import ADD, SET, SUB, Engine, _lib

pytestmark = pytest.mark.gpu


def _noalloc(p, A, B, Cm, op, stream):
    m, k = A.shape
    n = B.shape[1]
    return _lib.lib().hme_gemm_u32_dev_noalloc(p, m, n, k, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0),
                                               Cm.data_ptr(), Cm.stride(0), op, C.c_void_p(stream))


def _rand(g, shape, p):
    import torch

    return torch.randint(0, p, shape, dtype=torch.int64, device="cuda", generator=g).to(torch.int32)


@pytest.mark.parametrize("p,shape,op", [(65521, (1024, 1024, 1024), SET),
                                        (2147483629, (300, 200, 500), ADD),
                                        (251, (129, 700, 64), SUB),
                                        (16777213, (64, 96, 1200), SET),
                                        # k beyond one exact K chunk (8192 at four limbs): the chunk loop runs
                                        # twice, the second chunk accumulating on the first
                                        (2147483629, (64, 64, 9000), SET),
                                        (2147483629, (64, 64, 9000), SUB)])
def test_noalloc_matches_regular_entry_point_twice(p, shape, op):
    import torch

    m, n, k = shape
    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    st = torch.cuda.Stream()
    torch.cuda.set_stream(st)
    eng = Engine(0)
    eng.use_torch_stream()
    try:
        for call in range(2):  # two calls in a row, fresh inputs each time
            A, B, C0 = _rand(g, (m, k), p), _rand(g, (k, n), p), _rand(g, (m, n), p)
            want = C0.clone()
            eng.gemm_dev(p, A, B, want, op)
            eng.sync()
            got = C0.clone()
            torch.cuda.synchronize()
            rc = _noalloc(p, A, B, got, op, st.cuda_stream)
            assert rc == 0, _lib.lib().hme_last_error().decode()
            assert torch.equal(got, want), f"call {call}: allocation-free GEMM differs from hme_gemm_u32_dev"
    finally:
        eng.close()
        torch.cuda.set_stream(torch.cuda.default_stream())


def test_noalloc_rejects_oversized_product():
    import torch

    p, m, n, k = 2147483629, 4096, 4096, 4096  # 4-limb planes of 335 MB > 32 MiB
    A = torch.zeros((m, k), dtype=torch.int32, device="cuda")
    B = torch.zeros((k, n), dtype=torch.int32, device="cuda")
    Cm = torch.full((m, n), 7, dtype=torch.int32, device="cuda")
    rc = _noalloc(p, A, B, Cm, SET, 0)
    assert rc == _lib.HME_EINVAL
    assert "32 MiB" in _lib.lib().hme_last_error().decode()
    assert int(Cm[0, 0]) == 7  # nothing ran


def test_noalloc_refuses_stream_capture():
    """The entry point waits for its stream before it returns, which a stream
    being captured into a CUDA graph cannot do: it refuses the call up front
    and leaves the capture intact."""
    import torch

    p = 65521
    A = torch.ones((32, 32), dtype=torch.int32, device="cuda")
    B = torch.ones((32, 32), dtype=torch.int32, device="cuda")
    Cm = torch.zeros((32, 32), dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph, stream=st):
        Cm.add_(1)
        rc = _noalloc(p, A, B, Cm, SET, st.cuda_stream)
    assert rc == _lib.HME_EINVAL
    assert "capture" in _lib.lib().hme_last_error().decode()
    graph.replay()
    torch.cuda.synchronize()
    assert int(Cm[0, 0]) == 1  # the captured work ran; the refused call did not
