"""PyTorch fp32 reference of the library's 3D U-Net (test infrastructure only).

Same parameter layout as librtb200.so (per convolution: weights [cout][27][cin] with
tap = 9 (dz+1) + 3 (dy+1) + (dx+1), then bias [cout]; then head weights [3][16] and
bias [3]).  ``emulate_bf16`` reproduces where the kernels round to bf16: the stored
activations (every convolution output, pooled and upsampled tensors), the convolution
weights, and the pre-activation gradients that feed the tensor-core backward passes.
"""
import numpy as np
import torch
import torch.nn.functional as F

PLAN = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 48), (48, 48), (48, 64), (64, 64), (112, 48), (48, 48), (80, 32),
        (32, 32), (48, 16), (16, 16)]


def _bf(x):
    return x.to(torch.bfloat16).to(torch.float32)


class _RoundGrad(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return x.view_as(x)

    @staticmethod
    def backward(ctx, g):
        return _bf(g)


class _RoundVal(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return _bf(x)

    @staticmethod
    def backward(ctx, g):
        return g


def split_params(p):
    """Flat parameter vector -> list of (w [cout,27,cin], b [cout]) and (head_w [3,16], head_b [3])."""
    off = 0
    layers = []
    for cin, cout in PLAN:
        w = p[off:off + 27 * cin * cout].reshape(cout, 27, cin)
        off += 27 * cin * cout
        b = p[off:off + cout]
        off += cout
        layers.append((w, b))
    hw = p[off:off + 48].reshape(3, 16)
    off += 48
    hb = p[off:off + 3]
    off += 3
    assert off == p.numel()
    return layers, (hw, hb)


def _conv(x, w, b, emulate):
    # x [1, C, Z, Y, X]; w [cout, 27, cin] -> [cout, cin, kz, ky, kx]
    cout, _, cin = w.shape
    wk = w.reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)
    pre = F.conv3d(x, wk, b, padding=1)
    if emulate:
        pre = _RoundGrad.apply(pre)
    y = torch.relu(pre)
    return _RoundVal.apply(y) if emulate else y


def _pool(x, emulate):
    _, C, Z, Y, X = x.shape
    pz, py, px = Z % 2, Y % 2, X % 2
    xp = F.pad(x, (0, px, 0, py, 0, pz))
    ones = F.pad(torch.ones(1, 1, Z, Y, X, dtype=x.dtype), (0, px, 0, py, 0, pz))
    s = F.avg_pool3d(xp, 2) * 8
    n = F.avg_pool3d(ones, 2) * 8
    y = s / n
    return _RoundVal.apply(y) if emulate else y


def _up(x, shape):
    Z, Y, X = shape
    y = x.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)
    return y[:, :, :Z, :Y, :X]


def forward(p, inp, dims, emulate_bf16=True):
    """p: flat fp32 parameters (tensor, may require grad); inp: [V, 16] fp32; dims (X, Y, Z).
    Returns [V, 3]."""
    X, Y, Z = dims
    layers, (hw, hb) = split_params(p)
    if emulate_bf16:
        layers = [(_RoundVal.apply(w), b) for w, b in layers]
    x = inp.reshape(Z, Y, X, 16).permute(3, 0, 1, 2).unsqueeze(0)
    e = emulate_bf16
    a0 = _conv(x, *layers[0], e)
    e0 = _conv(a0, *layers[1], e)
    p1 = _pool(e0, e)
    a1 = _conv(p1, *layers[2], e)
    e1 = _conv(a1, *layers[3], e)
    p2 = _pool(e1, e)
    a2 = _conv(p2, *layers[4], e)
    e2 = _conv(a2, *layers[5], e)
    p3 = _pool(e2, e)
    a3 = _conv(p3, *layers[6], e)
    b3 = _conv(a3, *layers[7], e)
    d2a = _conv(torch.cat([_up(b3, e2.shape[2:]), e2], 1), *layers[8], e)
    d2 = _conv(d2a, *layers[9], e)
    d1a = _conv(torch.cat([_up(d2, e1.shape[2:]), e1], 1), *layers[10], e)
    d1 = _conv(d1a, *layers[11], e)
    d0a = _conv(torch.cat([_up(d1, e0.shape[2:]), e0], 1), *layers[12], e)
    d0 = _conv(d0a, *layers[13], e)
    feat = d0.squeeze(0).permute(1, 2, 3, 0).reshape(-1, 16)
    return feat @ hw.T + hb


def loss_and_grads(p_np, inp, tgt, dims, emulate_bf16=True):
    p = torch.tensor(p_np, dtype=torch.float32, requires_grad=True)
    out = forward(p, inp, dims, emulate_bf16)
    loss = ((out - tgt) ** 2).mean()
    loss.backward()
    return float(loss), p.grad.numpy().copy(), out.detach()
