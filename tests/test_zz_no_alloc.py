"""rt_compliance_noalloc: the allocation-free compliance entry point.

It serves callers that cannot call cudaMalloc (their device memory is owned by
their own pool, or allocation is barred while their solve loop runs), so it
takes caller-owned device vectors and keeps its scratch in a fixed array inside
the library.  The check: through the C ABI, two calls in a row agree with the
existing rt_compliance entry point on the same vectors.  This file is collected
last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import robtop_b200 as rb
from robtop_b200 import _capi as A
from robtop_b200 import configs

pytestmark = pytest.mark.gpu


def test_noalloc_compliance_matches_rt_compliance_twice():
    import torch

    cfg = configs.cantilever(24, 12, 12)
    ctx = rb.Context(0)
    G = rb.HierarchyGrid(ctx, rb.default_params(mode=cfg["mode"]))
    G.genFromBox(cfg["eact"])
    nv = G[0].nv
    n = 3 * nv
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(7)
    for call in range(2):
        u = rng.standard_normal(n)
        f = rng.standard_normal(n) * (call + 1)
        G[0].setDisplacement(u)
        G[0].setForce(f)
        c_ref = G[0].compliance()  # existing entry point (hierarchy-owned buffers)
        fd = torch.from_numpy(f).to(dev)
        ud = torch.from_numpy(u).to(dev)
        out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        st = A.lib().rt_compliance_noalloc(C.c_void_p(fd.data_ptr()), C.c_void_p(ud.data_ptr()), n,
                                           C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == A.RT_OK
        torch.cuda.synchronize(dev)
        c = float(out.item())
        assert abs(c - c_ref) <= 1e-12 * max(abs(c_ref), 1.0), (call, c, c_ref)
        assert abs(c - float(f @ u)) <= 1e-10 * np.sqrt(n) * max(abs(c_ref), 1.0)
    # n = 0 (only the final sum runs: 0.0), and a length whose partial-sum count (258) is above
    # the final kernel's 256-thread stride and not a multiple of it
    for n2 in (0, 257 * 4096 + 5):
        a = rng.standard_normal(max(n2, 1))
        b = rng.standard_normal(max(n2, 1))
        ad = torch.from_numpy(a).to(dev)
        bd = torch.from_numpy(b).to(dev)
        out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        st = A.lib().rt_compliance_noalloc(C.c_void_p(ad.data_ptr()), C.c_void_p(bd.data_ptr()), n2,
                                           C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == A.RT_OK
        torch.cuda.synchronize(dev)
        c = float(out.item())
        ref = float(a[:n2] @ b[:n2])
        assert abs(c - ref) <= 1e-10 * np.sqrt(max(n2, 1)) * max(abs(ref), 1.0), (n2, c, ref)
    # sizes beyond the scratch capacity are rejected before any kernel runs
    max_n = 65536 * 4096  # RT_NOALLOC_MAX_N in include/rtb200.h
    st = A.lib().rt_compliance_noalloc(C.c_void_p(fd.data_ptr()), C.c_void_p(ud.data_ptr()), max_n + 1,
                                       C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert st == A.RT_EINVAL
    G.close()
    ctx.close()
