"""Tensor-core (tcgen05) 3x3x3 convolution of the learned preconditioner against a plain
PyTorch fp32 reference (torch.nn.functional.conv3d on the CPU) on the same bf16 inputs."""
import ctypes as C

import numpy as np
import pytest
import torch

import robtop_b200 as rb

pytestmark = pytest.mark.gpu


def _to_torch_layout(a, X, Y, Z, Cn):
    # [V][C] channels-last (x fastest) -> [1, C, Z, Y, X]
    return a.reshape(Z, Y, X, Cn).permute(3, 0, 1, 2).unsqueeze(0)


def _ref_conv(inp, w, bias, X, Y, Z, cin, cout, relu):
    x = _to_torch_layout(inp.float().cpu(), X, Y, Z, cin)
    wt = w.float().cpu().reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)  # [cout][cin][kz][ky][kx]
    y = torch.nn.functional.conv3d(x, wt, bias.cpu() if bias is not None else None, padding=1)
    if relu:
        y = torch.relu(y)
    return y.squeeze(0).permute(1, 2, 3, 0).reshape(-1, cout)  # [V][cout]


@pytest.mark.parametrize("cin,cout,dims", [(16, 16, (19, 13, 11)), (48, 32, (9, 17, 10)), (112, 48, (8, 8, 7)),
                                           (32, 112, (16, 16, 3)), (64, 64, (40, 5, 6)), (16, 64, (21, 35, 19))])
@pytest.mark.parametrize("relu", [0, 1])
@pytest.mark.parametrize("variant", [1, 0])
def test_conv3_tc_matches_torch(cin, cout, dims, relu, variant):
    rb.lib().rt_unet_set_conv_variant(variant)
    X, Y, Z = dims
    V = X * Y * Z
    g = torch.Generator().manual_seed(cin * 1000 + cout + relu)
    inp = torch.randn(V, cin, generator=g).to(torch.bfloat16)
    w = (torch.randn(cout, 27, cin, generator=g) / np.sqrt(27 * cin)).to(torch.bfloat16)
    bias = torch.randn(cout, generator=g) * 0.1
    ref = _ref_conv(inp, w, bias, X, Y, Z, cin, cout, relu)
    ctx = rb.Context(0)
    di, dw, db = inp.cuda(), w.cuda(), bias.cuda()
    out = torch.zeros(V, cout, dtype=torch.float32, device="cuda")
    rb._capi.check(rb.lib().rt_unet_conv3(ctx.handle, C.c_void_p(di.data_ptr()), cin, cin, C.c_void_p(dw.data_ptr()),
                                          C.c_void_p(db.data_ptr()), cout, C.c_void_p(out.data_ptr()), cout, 1, relu,
                                          0, X, Y, Z), ctx.handle)
    got = out.cpu()
    # fp32 accumulation of bf16 products in a different order: relative 1e-5 of the output scale
    scale = ref.abs().max().item()
    assert (got - ref).abs().max().item() <= 2e-5 * scale + 1e-6
    # bf16 output with a row stride (the encoder writes into its decoder concat buffer)
    stride = cout + 16
    outb = torch.zeros(V, stride, dtype=torch.bfloat16, device="cuda")
    rb._capi.check(rb.lib().rt_unet_conv3(ctx.handle, C.c_void_p(di.data_ptr()), cin, cin, C.c_void_p(dw.data_ptr()),
                                          C.c_void_p(db.data_ptr()), cout, C.c_void_p(outb.data_ptr() + 32), stride,
                                          0, relu, 0, X, Y, Z), ctx.handle)
    gb = outb.cpu().float()
    assert torch.all(gb[:, :16] == 0)
    assert (gb[:, 16:] - ref.to(torch.bfloat16).float()).abs().max().item() <= 1e-2 * scale
    # accumulate into a float output
    acc = torch.ones(V, cout, dtype=torch.float32, device="cuda")
    rb._capi.check(rb.lib().rt_unet_conv3(ctx.handle, C.c_void_p(di.data_ptr()), cin, cin, C.c_void_p(dw.data_ptr()),
                                          None, cout, C.c_void_p(acc.data_ptr()), cout, 1, 0, 1, X, Y, Z), ctx.handle)
    ref_nb = _ref_conv(inp, w, None, X, Y, Z, cin, cout, 0)
    assert (acc.cpu() - 1.0 - ref_nb).abs().max().item() <= 2e-5 * scale + 1e-5
    rb.lib().rt_unet_set_conv_variant(1)
    ctx.close()


def test_conv3_rejects_bad_channels():
    ctx = rb.Context(0)
    buf = torch.zeros(1024, dtype=torch.bfloat16, device="cuda")
    st = rb.lib().rt_unet_conv3(ctx.handle, C.c_void_p(buf.data_ptr()), 24, 24, C.c_void_p(buf.data_ptr()), None, 16,
                                C.c_void_p(buf.data_ptr()), 16, 0, 0, 0, 4, 4, 4)
    assert st == rb._capi.RT_EINVAL
    ctx.close()


# ---------------------------------------------------------------------------
# the whole network: forward, loss and gradients against the fp32 reference
# ---------------------------------------------------------------------------
def test_unet_gradients_match_reference():
    import unet_ref
    from robtop_b200 import learned

    dims = (24, 20, 18)  # 27 voxels at the bottleneck level (3 x 3 x 3)
    V = dims[0] * dims[1] * dims[2]
    ctx = rb.Context(0)
    net = learned.UNet(ctx, *dims, seed=7)
    p = net.get_params()
    assert p.size == net.n_params() == 684851
    g = torch.Generator().manual_seed(3)
    inp = torch.randn(V, 16, generator=g)
    inp[:, 5:] = 0
    inp_b = inp.to(torch.bfloat16)
    tgt = torch.randn(V, 3, generator=g)
    out_gpu = net.forward(inp_b.cuda()).cpu()
    loss_ref, g_ref, out_ref = unet_ref.loss_and_grads(p, inp_b.float(), tgt, dims, emulate_bf16=True)
    # forward: bf16 storage of every activation; fp32 accumulation order differs
    assert (out_gpu - out_ref).abs().max().item() <= 2e-2 * out_ref.abs().max().item()
    loss, g_gpu = net.gradients(inp_b.cuda(), tgt.cuda())
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    # The pre-activation gradients are rounded to bf16 at every layer (as the tensor-core backward
    # consumes them) and ReLU masks of near-zero pre-activations can differ between the two
    # accumulation orders, so element-wise agreement is statistical: the whole gradient must agree
    # closely, each layer's direction must agree (a wrong tap order or transpose gives a cosine
    # near 0).
    rel_all = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    cos_all = float(g_gpu @ g_ref) / (np.linalg.norm(g_gpu) * np.linalg.norm(g_ref))
    assert rel_all < 5e-2 and cos_all > 0.999, (rel_all, cos_all)
    off = 0
    for cin, cout in unet_ref.PLAN + [(16, 3)]:
        n = 27 * cin * cout + cout if (cin, cout) != (16, 3) else 51
        a, b = g_gpu[off:off + n], g_ref[off:off + n]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        cos = float(a @ b) / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        assert rel < 0.2 and cos > 0.98, (cin, cout, rel, cos)
        off += n
    assert off == p.size
    net.close()
    ctx.close()


def test_unet_fp32_reference_agrees_with_emulated():
    # sanity of the reference itself: bf16 emulation changes the result only at bf16 level
    import unet_ref

    dims = (9, 8, 8)
    V = dims[0] * dims[1] * dims[2]
    ctx = rb.Context(0)
    from robtop_b200 import learned

    net = learned.UNet(ctx, *dims, seed=11)
    p = torch.tensor(net.get_params())
    inp = torch.randn(V, 16, generator=torch.Generator().manual_seed(5)).to(torch.bfloat16).float()
    a = unet_ref.forward(p, inp, dims, emulate_bf16=True)
    b = unet_ref.forward(p, inp, dims, emulate_bf16=False)
    assert (a - b).abs().max().item() <= 5e-2 * b.abs().max().item()
    net.close()
    ctx.close()
