"""The allocation-free 2-D DST entry point (ibfs_dst2d_noalloc) against the
existing handle-based transform (ibfs_apply_op, op 0) and against the
oracle's dst.

ibfs_dst2d_noalloc is for callers that cannot call cudaMalloc where they need
the transform: a driver whose memory pool owns all device memory, or a runtime
that keeps the CUDA allocator off its solver thread. Its intermediate product
lives in a fixed file-scope device array and it takes device pointers that the
caller already owns. This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import ibfs_capi as C
import oracle as O

TOL = 1e-12  # same bar as the handle-based transform in test_gpu_parity


def _noalloc(x_dev, y_dev, m, n, stream):
    return C.lib().ibfs_dst2d_noalloc(ctypes.c_void_p(x_dev.data_ptr()), ctypes.c_void_p(y_dev.data_ptr()),
                                      m, n, ctypes.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("m,n", [(64, 48), (400, 400), (512, 512)])
def test_noalloc_dst_matches_handle_dst_and_oracle(m, n):
    import torch
    xb, yb = O.circle(4.0 / m, 1.0, 0.0, 0.0)
    g = C.Solver(C.make_params(m, n, 0.01, 100.0, 2), (xb, yb))
    oc = O.Case(O.make_params(m, n, 0.01, 100.0, 2), xb, yb)
    rng = np.random.default_rng(11)
    ns = (m - 1) * (n - 1)
    stream = torch.cuda.current_stream().cuda_stream
    y_dev = torch.empty(ns, dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row share the static scratch
        x = rng.standard_normal(ns) * (1.0 + call)
        ref = g.apply_op(0, x)
        x_dev = torch.from_numpy(x).to("cuda")
        rc = _noalloc(x_dev, y_dev, m, n, stream)
        assert rc == C.OK, C.lib().ibfs_last_error(None).decode()
        torch.cuda.synchronize()
        y = y_dev.cpu().numpy()
        err = np.abs(y - ref).max() / np.abs(ref).max()
        assert err < TOL, (call, err)
        orc = oc.dst(x)
        err_o = np.abs(y - orc).max() / np.abs(orc).max()
        assert err_o < TOL, (call, err_o)
    g.close()


@pytest.mark.gpu
def test_noalloc_rejects_oversize():
    import torch
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = _noalloc(x, x, 1024, 64, torch.cuda.current_stream().cuda_stream)
    assert rc == C.ERR_ARG
    assert "511" in C.lib().ibfs_last_error(None).decode()
