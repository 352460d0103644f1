"""The method of moving asymptotes (optimization/mma_t.{h,cpp,cu}) on the device against the
oracle's restatement (oracle/or_mma.c): the same steps from the same FP32 gradients, and the
known optimum of a separable problem; then the MMA density loop of TestSuit::testtest2011
(utils/test_utils.cpp:1750-1800) for three iterations on a small worst-case box, device
against oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from gpu_common import CONFIGS, E, NU, P, build_pair
from robtop_b200.mma import MMA

pytestmark = pytest.mark.gpu


def _separable(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.5, 2.0, n), 0.3


def _grads(c, x, V):
    """min sum c_j / x_j / n  s.t.  1e3 (mean(x) - V) <= 0 (the reference's constraint scaling)."""
    n = c.size
    df = (-c / x ** 2 / n).astype(np.float32)
    dg = np.full(n, 1e3 / n, np.float32)
    return df, dg, 1e3 * (x.mean() - V)


def test_mma_steps_match_oracle_and_reach_the_optimum():
    """12 steps of the device's MMA and the oracle's from the same start, each from the FP32
    gradients at its own design: designs within 1e-6 and multipliers within 1e-6 relative after
    every step (the two sum in different orders, and a variable whose step is near zero can take
    the other asymptote factor, 0.7 or 1.2, in the next step); the device then runs to the
    separable problem's optimum x_j = V n sqrt(c_j) / sum sqrt(c) (all inside the bounds here)
    to 1e-6."""
    n = 200_003  # not a multiple of the block size
    c, V = _separable(n, 1)
    ctx = rb.Context(0)
    m = MMA(ctx, n, 0.01, 1.0)
    o = O.MMA(n, 0.01, 1.0)
    try:
        assert np.array_equal(m.x, o.x)
        for it in range(60):
            df, dg, g = _grads(c, m.x, V)
            m.update(df, dg, g)
            if it < 12:
                df_o, dg_o, g_o = _grads(c, o.x, V)
                lam_o = o.update(df_o.astype(np.float64), dg_o.astype(np.float64), g_o)
                assert np.abs(m.x - o.x).max() <= 1e-6, it
                assert abs(m.lam - lam_o) <= 1e-6 * max(abs(lam_o), 1e-300), (it, m.lam, lam_o)
        xs = V * n * np.sqrt(c) / np.sqrt(c).sum()
        assert np.abs(m.x - xs).max() <= 1e-6
        assert abs(m.x.mean() - V) <= 1e-9
        assert m.evaluations > 0
    finally:
        m.close()
        ctx.close()


def test_mma_bounds_arrays_and_errors():
    """Per-variable bounds keep the design inside them; a non-finite constraint value is
    RT_ENAN; bounds with xmax <= xmin are refused."""
    n = 4096
    rng = np.random.default_rng(3)
    lo = rng.uniform(0.0, 0.3, n)
    hi = lo + rng.uniform(0.1, 0.7, n)
    ctx = rb.Context(0)
    m = MMA(ctx, n, lo, hi)
    try:
        assert np.allclose(m.x, 0.5 * (lo + hi))
        c = rng.uniform(0.5, 2.0, n)
        for _ in range(10):
            df, dg, g = _grads(c, m.x, 0.25)
            m.update(df, dg, g)
            assert np.all(m.x >= lo - 1e-15) and np.all(m.x <= hi + 1e-15)
        with pytest.raises(RuntimeError):
            m.update(df, dg, float("nan"))
    finally:
        m.close()
    with pytest.raises(RuntimeError):
        MMA(ctx, n, hi, lo)
    ctx.close()


def test_mma_density_loop_against_oracle():
    """Three iterations of the testtest2011 loop on the 20x16x12 worst-case box: densities from
    the design, stencil update, worst-case load by Lanczos (k = 8, inner solves to 1e-10), its
    displacement, filtered sensitivity times 1e5, MMA step with the volume constraint
    1e3 (vol - 0.4) and gradient 1e3 / n_active on the active elements, each side from its own
    design.  The device's and the oracle's eigenvalues agree to 1e-6 and their designs to 1e-4
    after every step."""
    import torch

    cfg = CONFIGS["worstcase"]()
    ctx, G, H = build_pair(cfg)
    nz, ny, nx = cfg["eact"].shape
    eact = np.ascontiguousarray(cfg["eact"].ravel(), np.uint8)
    ne, n_act = eact.size, int(eact.sum())
    ln = np.ascontiguousarray(cfg["load_nodes"], np.int32)
    normals = np.ascontiguousarray(cfg["normals"], np.float64)
    dv = np.where(eact != 0, 1e3 / n_act, 0.0).astype(np.float32)
    m = MMA(ctx, ne, 1e-3, 1.0)
    o = O.MMA(ne, 1e-3, 1.0)
    K, TOL = 8, 1e-10
    sens = torch.empty(ne, dtype=torch.float32, device="cuda")
    try:
        for it in range(3):
            # device
            m.set_density(G)
            G.update_stencil()
            xg = m.x
            vol_g = float(xg[eact != 0].sum()) / n_act
            lam_g, _ = G.worst_case(rb.WORST_LANCZOS, K, TOL, seed=200 + it)
            rb._capi.check(rb.lib().rt_sensitivity(G.handle, 1), ctx.handle)
            rb._capi.check(rb.lib().rt_get_dev(G.handle, rb._capi.FIELD_SENS, 0, C.c_void_p(sens.data_ptr())),
                           ctx.handle)
            ctx.sync()
            s_g = sens.cpu().numpy()
            m.update(s_g * np.float32(1e5), dv, 1e3 * (vol_g - 0.4))
            # oracle
            rho_o = np.where(eact != 0, o.x, 0).astype(np.float32)
            Ho = O.Hierarchy(cfg["eact"], rho_o.reshape(cfg["eact"].shape), cfg["vfix"], p=P, E=E, nu=NU)
            Ho.update_stencil()
            nv = Ho.arrs[0]["u"].size // 3
            work = np.zeros((K + 1) * 3 * ln.size + 10 * 3 * nv)
            lam, ritz = np.zeros(1), np.zeros(3 * nv)
            O.lib().or_lanczos(Ho.LA, Ho.nlev, O.ptr(Ho.KE), O.SMOOTH_SGS, 1, 1, 0.6, ln.size, O.ptr(ln),
                               O.ptr(normals), 0, 0, None, 200 + it, K, TOL, 2000, O.ptr(lam), O.ptr(ritz),
                               O.ptr(work))
            assert abs(lam_g - lam[0]) <= 1e-6 * lam[0], (it, lam_g, lam[0])
            x, _, _ = Ho.pcg(ritz, tol=TOL, maxit=2000)
            s = np.zeros(ne, np.float32)
            O.lib().or_sensitivity(nx, ny, nz, O.ptr(eact), O.ptr(rho_o), P, O.ptr(Ho.KE), O.ptr(x), O.ptr(s))
            fs = np.zeros_like(s)
            O.lib().or_filter(nx, ny, nz, O.ptr(eact), 2.0, O.ptr(s), O.ptr(fs))
            vol_o = float(o.x[eact != 0].sum()) / n_act
            o.update((fs * np.float32(1e5)).astype(np.float64), dv.astype(np.float64), 1e3 * (vol_o - 0.4))
            assert np.abs(m.x - o.x)[eact != 0].max() <= 1e-4, it
        assert np.abs(m.x - 0.5005)[eact != 0].max() > 1e-3  # the design moved from the start
    finally:
        m.close()
        G.close()
        ctx.close()


def test_mma_optimisation_loop_through_the_module():
    """robtop_b200.mma.optimization_mma (TestSuit::testtest2011's loop) on the 24x12x12
    cantilever built through the optimization module: four MMA iterations with the worst-case
    eigenvalue by Lanczos; the eigenvalues are finite and positive and the design's volume
    moves from the middle of the bounds towards the 0.4 target."""
    from robtop_b200 import mma as M
    from robtop_b200 import optimization as opt

    opt.setParameters(0.4, 0.0, 0.03, 2, 0.5, 3.0, 1e-3, 32, 1e6, 0.4)
    opt.setWorkMode("wsff")
    nx, ny, nz, R = 24, 12, 12, 32
    opt.setBoundaryCondition(lambda p: p[0] == 0.0, lambda p: p[0] == nx and p[2] == 0.0,
                             lambda p: (0.0, 0.0, -1.0))
    bits = np.zeros((R ** 3 + 31) // 32, np.uint32)
    for z in range(nz):
        for y in range(ny):
            t = np.arange(nx) + R * (y + R * z)
            np.bitwise_or.at(bits, t >> 5, (np.uint32(1) << (t & 31).astype(np.uint32)))
    opt.buildGrids(bits, R)
    opt.uploadTemplateMatrix()
    rec = M.optimization_mma(max_iter=4, worst=lambda: opt.worstCaseLanczos(8, 1e-8, seed=3))
    assert len(rec) == 4 and all(np.isfinite(c) and c > 0 for c in rec)
    G = opt.getGrids()
    eact = G[0].getEact() != 0
    vol = float(G[0].getRho()[eact].mean())
    assert vol < 0.5005 - 1e-3 and vol > 0.3
