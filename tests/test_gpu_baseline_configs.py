"""Parity on the benchmark configurations themselves, not only on the small boxes of the other
parity tests.

* The small cantilever (64x32x32 elements, uniform density 0.4, x = 0 clamped, total load 1 in
  -z over the bottom edge of the x = 64 face): the FP64 V-cycle PCG with 2 + 2 damped block
  Jacobi sweeps to 1e-6, and one OC step (sensitivity, filter radius 2, move 0.03, damping
  0.5, volume 0.4), on the GPU and in the oracle.  With the specified omega = 0.6 both stall
  (lambda_max(D^-1 K) is above 2 / 0.6 on this box); both must report it the same way.
* The 128x128x64 worst-case box: the largest eigenvalue of the load-space compliance operator
  by Lanczos (k = 16, start vector seed 100), in the plain FP64 form and in the mixed form,
  against the oracle's value stored in tests/golden/c2_lanczos.npz (made by
  tests/golden/make_c2_lanczos.py with inner solves to 1e-9): eigenvalue within 1e-5, and the
  Ritz load on the top face parallel to the oracle's.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from robtop_b200 import configs

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
E, NU, P = 1e6, 0.4, 3.0


def _c1(omega):
    cfg = configs.cantilever(64, 32, 32)
    ctx = rb.Context(0)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=E, poisson_ratio=NU, power_penalty=P, min_rho=1e-3,
                          precision=rb.FP64, smoother=rb.SMOOTH_JACOBI, pre_sweeps=2, post_sweeps=2,
                          jacobi_omega=omega, volume_ratio=0.4, design_step=0.03, damp_ratio=0.5, filter_radius=2.0)
    G = rb.HierarchyGrid(ctx, p)
    G.genFromBox(cfg["eact"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    G.update_stencil()
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=P, E=E, nu=NU)
    H.set_weights(G[0].getPenalty())
    H.update_stencil()
    return cfg, ctx, G, H


def test_c1_cantilever_solve_and_oc_step():
    cfg, ctx, G, H = _c1(0.5)
    try:
        b = np.ascontiguousarray(cfg["fload"].ravel(), np.float64)
        G[0].setForce(b)
        G[0].reset_displacement()
        info = G.pcg(1e-6, 500)
        assert info.status == 0 and info.rel_residual <= 1e-6
        u = G[0].getDisplacement()
        xo, it_o, rr_o = H.pcg(b, tol=1e-6, maxit=500, smoother=O.SMOOTH_JACOBI, npre=2, npost=2, omega=0.5)
        assert rr_o <= 1e-6
        # same method, same operator: the iteration counts agree and so do the solutions
        assert abs(info.iterations - it_o) <= 1, (info.iterations, it_o)
        c, co = float(b @ u), float(b @ xo)
        assert abs(c - co) <= 1e-6 * abs(co), (c, co)
        assert np.linalg.norm(u - xo) <= 1e-5 * np.linalg.norm(xo)
        # one OC step from the same displacement
        nz, ny, nx = cfg["eact"].shape
        eact = np.ascontiguousarray(cfg["eact"].ravel(), np.uint8)
        rho = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
        G[0].setDisplacement(xo)
        rb._capi.check(rb.lib().rt_sensitivity(G.handle, 0), ctx.handle)
        G[0].filterSensitivity(2.0)
        lam, trials = C.c_float(), C.c_int()
        rb._capi.check(rb.lib().rt_oc_update(G.handle, 0.4, C.byref(lam), C.byref(trials)), ctx.handle)
        rho_g = G[0].getRho()
        s = np.zeros(rho.size, np.float32)
        O.lib().or_sensitivity(nx, ny, nz, O.ptr(eact), O.ptr(rho), P, O.ptr(H.KE), O.ptr(xo), O.ptr(s))
        fs = np.zeros_like(s)
        O.lib().or_filter(nx, ny, nz, O.ptr(eact), 2.0, O.ptr(s), O.ptr(fs))
        rho_o, tmp = rho.copy(), np.zeros_like(rho)
        its = np.zeros(1, np.int32)
        O.lib().or_oc_update(rho.size, O.ptr(eact), None, O.ptr(rho_o), O.ptr(fs), 0.4, 0.03, 0.5, 1e-3,
                             int(eact.sum()), O.ptr(its), O.ptr(tmp))
        assert np.abs(rho_g - rho_o).max() <= 1e-4
        assert np.abs(rho_g - rho).max() > 1e-3  # the step moved the design
    finally:
        G.close()
        ctx.close()


def test_c1_specified_omega_stalls_in_both():
    """omega = 0.6 amplifies the top of the spectrum of D^-1 K on this box: neither the GPU nor
    the oracle reaches 1e-6 in 300 iterations, and they stall at the same level."""
    cfg, ctx, G, H = _c1(0.6)
    try:
        assert G.smoother_lmax(0) > 2.0 / 0.6
        b = np.ascontiguousarray(cfg["fload"].ravel(), np.float64)
        G[0].setForce(b)
        G[0].reset_displacement()
        info = G.pcg(1e-6, 300)
        _, it_o, rr_o = H.pcg(b, tol=1e-6, maxit=300, smoother=O.SMOOTH_JACOBI, npre=2, npost=2, omega=0.6)
        assert info.rel_residual > 1e-6 and rr_o > 1e-6
        assert 0.1 < info.rel_residual / rr_o < 10.0, (info.rel_residual, rr_o)
    finally:
        G.close()
        ctx.close()


GOLDEN = os.path.join(HERE, "golden", "c2_lanczos.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="tests/golden/c2_lanczos.npz not generated")
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_c2_worst_case_eigenvalue_against_golden(form):
    g = np.load(GOLDEN)
    nx, ny, nz = (int(v) for v in g["dims"])
    cfg = configs.worst_case_box(nx, ny, nz, seed=int(g["seed"]))
    ctx = rb.Context(0)
    kw = dict(precision=rb.FP64, smoother=rb.SMOOTH_SGS, pre_sweeps=1, post_sweeps=1)
    if form == "mixed":
        kw = dict(precision=rb.FP32, smoother=rb.SMOOTH_CHEBY, pre_sweeps=2, post_sweeps=2, coarse_sweeps=8)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=E, poisson_ratio=NU, power_penalty=P, min_rho=1e-3, **kw)
    G = rb.HierarchyGrid(ctx, p)
    try:
        G.genFromBox(cfg["eact"])
        G[0].setRho(cfg["rho"].ravel())
        G.set_support(cfg["vfix"])
        G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
        G.update_stencil()
        lam, info = G.worst_case(rb.WORST_LANCZOS, int(g["k"]), 1e-6, seed=int(g["start"]))
        assert abs(lam - float(g["lam"])) <= 1e-5 * abs(float(g["lam"])), (lam, float(g["lam"]))
        f = G[0].getForce()
        nv = G[0].nv
        ln = g["load_nodes"]
        assert np.array_equal(ln, cfg["load_nodes"])
        load = np.stack([f[c * nv + ln] for c in range(3)])
        ref = g["load"]
        cos = abs(float(np.sum(load * ref))) / (np.linalg.norm(load) * np.linalg.norm(ref))
        assert cos >= 1 - 1e-4, cos
    finally:
        G.close()
        ctx.close()


def test_c5_loop_checked_against_oracle_at_reduced_size():
    """C5's loop (arch domain with the tunnel and support pads, wscf top-face load, V 0.4, R 2,
    move 0.06, eta 0.5, p 3) at 63x32x32 elements, 12 OC iterations (rt_oc_iteration: Lanczos
    k = 16, inner solves to 1e-6) in the mixed form (FP32 Chebyshev(2) cycles, W below level 1).
    Every 4 iterations the design's worst-case eigenvalue and the compliance of a fixed unit
    top-face load are checked against the FP64 oracle on the same densities: eigenvalue within
    1e-5, compliance within 1e-6.  (At 511x256x256 the oracle would take about 40 minutes per
    check on the host; the bench's c5oc40 workload checks against the plain FP64 GPU path.)"""
    cfg = configs.arch(63, 32, 32, tunnel=12, pad=2)
    ctx = rb.Context(0)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=E, poisson_ratio=NU, power_penalty=P, min_rho=1e-3,
                          precision=rb.FP32, smoother=rb.SMOOTH_CHEBY, pre_sweeps=2, post_sweeps=2,
                          volume_ratio=0.4, design_step=0.06, damp_ratio=0.5, filter_radius=2.0)
    p.cycle_gamma = 2
    G = rb.HierarchyGrid(ctx, p)
    ln = np.ascontiguousarray(cfg["load_nodes"], np.int32)
    normals = np.ascontiguousarray(cfg["normals"], np.float64)
    try:
        G.genFromBox(cfg["eact"])
        G[0].setRho(cfg["rho"].ravel())
        G.set_support(cfg["vfix"])
        G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
        nv = G[0].nv
        fload = np.zeros(3 * nv)
        fload[2 * nv + ln] = 1.0 / np.sqrt(ln.size)
        lam_c = C.c_double()
        checks = 0
        for it in range(1, 13):
            rb._capi.check(rb.lib().rt_oc_iteration(G.handle, rb.WORST_LANCZOS, 16, 1e-6, 7, 0.4, C.byref(lam_c)),
                           ctx.handle)
            if it % 4:
                continue
            G.update_stencil()
            lam_g, _ = G.worst_case(rb.WORST_LANCZOS, 16, 1e-6, seed=7)
            G[0].setForce(fload)
            G[0].reset_displacement()
            info = G.pcg(1e-8, 2000)
            assert info.status == 0
            c_g = float(fload @ G[0].getDisplacement())
            rho = G[0].getRho().reshape(cfg["eact"].shape)
            H = O.Hierarchy(cfg["eact"], rho, cfg["vfix"], p=P, E=E, nu=NU)
            H.update_stencil()
            nvo = H.arrs[0]["u"].size // 3
            work = np.zeros(17 * 3 * ln.size + 10 * 3 * nvo)
            lo = np.zeros(1)
            O.lib().or_lanczos(H.LA, H.nlev, O.ptr(H.KE), O.SMOOTH_SGS, 1, 1, 0.6, ln.size, O.ptr(ln),
                               O.ptr(normals), 1, 0, None, 7, 16, 1e-8, 3000, O.ptr(lo), None, O.ptr(work))
            assert abs(lam_g - lo[0]) <= 1e-5 * lo[0], (it, lam_g, lo[0])
            xo, _, rr = H.pcg(fload, tol=1e-10, maxit=3000)
            assert rr <= 1e-10
            c_o = float(fload @ xo)
            assert abs(c_g - c_o) <= 1e-6 * abs(c_o), (it, c_g, c_o)
            checks += 1
        assert checks == 3
    finally:
        G.close()
        ctx.close()
