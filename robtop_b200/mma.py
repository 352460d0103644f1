"""The method of moving asymptotes as an alternative density update (optimization/mma_t.h:159-273,
optimization/mma_t.cpp:18-51), on the device through ``librtb200.so``.

``MMA(ctx, n, xmin, xmax)`` mirrors ``MMA::mma_t(n, 1)`` + ``init(lower, upper)``;
``update(df, dg, g)`` takes one step for ``min f0 s.t. f1 <= 0`` and returns the reference's
stop flag; ``x`` is the design.  ``optimization_mma`` is the loop of TestSuit::testtest2011
(utils/test_utils.cpp:1750-1800): densities from the design, stencil update, worst-case
compliance, filtered sensitivity scaled by 1e5, volume constraint scaled by 1e3.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A


def _device_f32(v, n):
    """A CUDA float32 tensor of n values (torch tensors on the device pass through)."""
    import torch

    if isinstance(v, torch.Tensor):
        t = v.detach()
        if not t.is_cuda or t.dtype != torch.float32 or not t.is_contiguous():
            t = t.to(device="cuda", dtype=torch.float32).contiguous()
    else:
        t = torch.as_tensor(np.ascontiguousarray(v, np.float32), device="cuda")
    if t.numel() != n:
        raise ValueError(f"expected {n} values, got {t.numel()}")
    torch.cuda.current_stream().synchronize()  # the library reads it on its own stream
    return t


class MMA:
    """MMA::mma_t for one constraint; bounds are arrays of n values or scalars."""

    def __init__(self, ctx, n, xmin=0.0, xmax=1.0):
        self.ctx = ctx
        self.n = int(n)
        h = C.c_void_p()
        if np.ndim(xmin) == 0 and np.ndim(xmax) == 0:
            st = A.lib().rt_mma_create(ctx.handle, self.n, None, None, float(xmin), float(xmax), C.byref(h))
        else:
            lo = np.ascontiguousarray(np.broadcast_to(np.asarray(xmin, np.float64), (self.n,)))
            hi = np.ascontiguousarray(np.broadcast_to(np.asarray(xmax, np.float64), (self.n,)))
            st = A.lib().rt_mma_create(ctx.handle, self.n, lo.ctypes.data_as(C.c_void_p),
                                       hi.ctypes.data_as(C.c_void_p), 0.0, 0.0, C.byref(h))
        A.check(st, ctx.handle)
        self.handle = h
        self.lam = 0.0
        self.dxnorm = 0.0

    def update(self, df, dg, g):
        """One step from the objective gradient df, the constraint gradient dg (n values each,
        used as FP32 as the reference's Scalar) and the constraint value g; True once the
        reference's stop rule fires."""
        d0, d1 = _device_f32(df, self.n), _device_f32(dg, self.n)
        stop, lam, dxn = C.c_int(), C.c_double(), C.c_double()
        A.check(A.lib().rt_mma_update(self.handle, C.c_void_p(d0.data_ptr()), C.c_void_p(d1.data_ptr()), float(g),
                                      C.byref(stop), C.byref(lam), C.byref(dxn)), self.ctx.handle)
        self.lam, self.dxnorm = lam.value, dxn.value
        return bool(stop.value)

    @property
    def x(self):
        out = np.empty(self.n)
        A.check(A.lib().rt_mma_get_x(self.handle, out.ctypes.data_as(C.c_void_p)), self.ctx.handle)
        return out

    def set_density(self, G):
        """setDensity(mma.get_x()): the design becomes the finest level's densities."""
        A.check(A.lib().rt_mma_set_density(self.handle, G.handle), self.ctx.handle)

    @property
    def evaluations(self):
        return int(A.lib().rt_mma_evaluations(self.handle))

    def close(self):
        if self.handle:
            A.lib().rt_mma_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def optimization_mma(max_iter=100, worst=None, vol_scale=1e3, sens_scale=1e5):
    """TestSuit::testtest2011 (utils/test_utils.cpp:1750-1800) on the module's grids: MMA on the
    densities with bounds [min_rho, 1], constraint volScale (vol - volume_ratio) with gradient
    volScale / n_active on the active elements, objective gradient the filtered sensitivity of
    the worst-case compliance times sensScale.  Returns the worst-case compliance of each
    iteration; stops early when the reference's MMA stop rule fires."""
    import torch

    from . import optimization as opt

    G = opt.getGrids()
    worst = worst or opt.modifiedPM
    ne = G[0].ne
    eact = torch.as_tensor(np.ascontiguousarray(G[0].getEact(), np.uint8), device="cuda").to(torch.float64)
    n_act = float(eact.sum().item())
    m = MMA(opt._ctx(), ne, opt.params.min_rho, 1.0)
    dv = (eact * (vol_scale / n_act)).to(torch.float32)
    sens = torch.empty(ne, dtype=torch.float32, device="cuda")
    rec = []
    try:
        for _ in range(max_iter):
            m.set_density(G)
            opt.update_stencil()
            x = torch.as_tensor(m.x, device="cuda")
            vol = float((x * eact).sum().item()) / n_act
            c = worst()
            rec.append(c)
            opt.computeSensitivity()
            A.check(A.lib().rt_get_dev(G.handle, A.FIELD_SENS, 0, C.c_void_p(sens.data_ptr())), opt._ctx().handle)
            torch.cuda.synchronize()
            if m.update(sens * sens_scale, dv, vol_scale * (vol - opt.params.volume_ratio)):
                break
    finally:
        m.close()
    return rec
