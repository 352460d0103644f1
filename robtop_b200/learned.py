"""Learned preconditioner: the 3D U-Net of ``librtb200.so`` (tensor-core convolutions,
BF16 activations, FP32 accumulation), its training-sample harvest from the solver, its
training loop, and its use inside MG-PCG as z = Vcycle(r) + N(rho, r).

Device buffers are torch CUDA tensors (plumbing only); every kernel is the library's.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check


def _vp(t):
    """Device pointer of a torch CUDA tensor for the library.  The library runs on its context's
    own stream, so torch's pending work on the tensor (the copy or fill that made it) is waited
    for first."""
    import torch

    torch.cuda.current_stream(t.device).synchronize()
    return C.c_void_p(t.data_ptr())


class UNet:
    """rt_unet over an X x Y x Z node box (the finest node box of the hierarchies it serves)."""

    def __init__(self, ctx, X, Y, Z, seed=0):
        self.ctx = ctx
        self.dims = (int(X), int(Y), int(Z))
        self.V = int(X) * int(Y) * int(Z)
        self._u = C.c_void_p()
        check(A.lib().rt_unet_create(ctx.handle, int(X), int(Y), int(Z), int(seed), C.byref(self._u)), ctx.handle)

    @classmethod
    def for_grid(cls, G, seed=0):
        L = G[0]
        return cls(G.ctx, L.nx + 1, L.ny + 1, L.nz + 1, seed)

    @property
    def handle(self):
        return self._u

    def _c(self, st):
        return check(st, self.ctx.handle)

    def n_params(self):
        return int(A.lib().rt_unet_n_params(self._u))

    def get_params(self):
        p = np.zeros(self.n_params(), np.float32)
        self._c(A.lib().rt_unet_get_params(self._u, p.ctypes.data_as(C.c_void_p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params()
        self._c(A.lib().rt_unet_set_params(self._u, p.ctypes.data_as(C.c_void_p)))

    @property
    def output_scale(self):
        return float(A.lib().rt_unet_output_scale(self._u))

    @output_scale.setter
    def output_scale(self, v):
        self._c(A.lib().rt_unet_set_output_scale(self._u, float(v)))

    def forward(self, inp):
        """inp: torch bf16 CUDA [V, 16] -> torch float32 CUDA [V, 3]."""
        import torch

        out = torch.empty(self.V, 3, dtype=torch.float32, device=inp.device)
        self._c(A.lib().rt_unet_forward(self._u, _vp(inp.contiguous()), _vp(out)))
        self.ctx.sync()  # out is written on the library's stream
        return out

    def gradients(self, inp, tgt):
        """Loss and FP32 parameter gradients of one sample (no update)."""
        loss = C.c_double()
        g = np.zeros(self.n_params(), np.float32)
        self._c(A.lib().rt_unet_gradients(self._u, _vp(inp.contiguous()), _vp(tgt.contiguous()), C.byref(loss),
                                          g.ctypes.data_as(C.c_void_p)))
        return loss.value, g

    def train_step(self, inp, tgt, lr):
        """One Adam step on a batch: inp [B, V, 16] bf16, tgt [B, V, 3] float32 (CUDA)."""
        loss = C.c_double()
        self._c(A.lib().rt_unet_train_step(self._u, int(inp.shape[0]), _vp(inp.contiguous()),
                                           _vp(tgt.contiguous()), float(lr), C.byref(loss)))
        return loss.value

    def close(self):
        if self._u:
            A.lib().rt_unet_destroy(self._u)
            self._u = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def harvest(G, net, k_iter, seed):
    """One (input, target) training sample from hierarchy G (rt_unet_harvest)."""
    import torch

    inp = torch.empty(net.V, 16, dtype=torch.bfloat16, device="cuda")
    tgt = torch.empty(net.V, 3, dtype=torch.float32, device="cuda")
    check(A.lib().rt_unet_harvest(G.handle, net.handle, int(k_iter), int(seed), _vp(inp), _vp(tgt)), G.ctx.handle)
    G.ctx.sync()  # inp and tgt are written on the library's stream
    return inp, tgt


def attach(G, net, fallback_ratio=1.0, post_sweeps=0):
    """Use the network inside G's PCG (z = Vcycle(r) + N(rho, r, Vcycle(r))); net=None detaches.
    An iteration whose residual norm does not drop below ``fallback_ratio`` x the previous one
    switches the correction off until the next stencil update.  ``post_sweeps`` finest-level
    smoothing steps follow each correction."""
    check(A.lib().rt_hier_set_learned(G.handle, net.handle if net is not None else None, float(fallback_ratio)),
          G.ctx.handle)
    check(A.lib().rt_hier_set_learned_post(G.handle, int(post_sweeps)), G.ctx.handle)


def stats(G):
    """(corrections run since attach, whether the gate has switched the network off for this design)"""
    n = C.c_longlong()
    off = C.c_int()
    check(A.lib().rt_hier_learned_stats(G.handle, C.byref(n), C.byref(off)), G.ctx.handle)
    return int(n.value), bool(off.value)


def forward_seconds(net, reps=3):
    """Device time of one network application on the context stream (the forward pass on the
    network's own input buffer; each call synchronises the stream)."""
    import time

    check(A.lib().rt_unet_forward(net.handle, None, None), net.ctx.handle)
    t0 = time.perf_counter()
    for _ in range(reps):
        check(A.lib().rt_unet_forward(net.handle, None, None), net.ctx.handle)
    return (time.perf_counter() - t0) / reps


def cost_aware_ratio(plain_iterations, plain_rel_residual, plain_seconds, net_seconds):
    """Fallback ratio under which a learned iteration pays for itself.  The plain V-cycle PCG
    reduced the residual by q = rel_res^(1/its) per iteration in plain_seconds / its each; an
    iteration with the network costs c = (that + net_seconds) / that as much, so it must reduce
    the residual by q^c to reach the tolerance no later."""
    its = max(int(plain_iterations), 1)
    q = float(plain_rel_residual) ** (1.0 / its)
    t_it = float(plain_seconds) / its
    c = (t_it + float(net_seconds)) / t_it
    return q ** c


def train(net, samples, steps, batch=4, lr=1e-3, seed=0):
    """Adam on random batches of (input, target) samples; returns the loss history."""
    import torch

    rng = np.random.default_rng(seed)
    ins = torch.stack([s[0] for s in samples])
    tgts = torch.stack([s[1] for s in samples])
    losses = []
    for _ in range(steps):
        idx = torch.as_tensor(rng.choice(len(samples), size=min(batch, len(samples)), replace=False),
                              device=ins.device)
        losses.append(net.train_step(ins[idx], tgts[idx], lr))
    return losses


def crops(inp, tgt, dims, crop, n, rng):
    """n random crops (each a box of ``crop`` node dims) of one full-box sample, as contiguous
    [v, 16] / [v, 3] tensors; the residual scaling of the full box is kept."""
    X, Y, Z = dims
    cx, cy, cz = crop
    a = inp.view(Z, Y, X, 16)
    t = tgt.view(Z, Y, X, 3)
    out = []
    for _ in range(n):
        x0 = int(rng.integers(0, X - cx + 1))
        y0 = int(rng.integers(0, Y - cy + 1))
        z0 = int(rng.integers(0, Z - cz + 1))
        out.append((a[z0:z0 + cz, y0:y0 + cy, x0:x0 + cx].reshape(-1, 16).contiguous(),
                    t[z0:z0 + cz, y0:y0 + cy, x0:x0 + cx].reshape(-1, 3).contiguous()))
    return out


def transfer(src, dst):
    """Copy the weights and the output unit of one network to another (any box)."""
    dst.set_params(src.get_params())
    dst.output_scale = src.output_scale
