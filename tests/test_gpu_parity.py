"""GPU parity: every kernel of the hot path, called through the C ABI, against the
CPU oracle on the same seeded inputs.

Tolerances: integer / occupancy / index work is bit-exact; FP64 kernels agree
to 1e-11 relative (max-norm, summation order differs); iterative solves agree
to the stated solver tolerance; FP32 paths are judged on the FP64 residual.
"""
import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from gpu_common import CONFIGS, build_pair, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11


@pytest.fixture(scope="module", params=sorted(CONFIGS))
def pair(request):
    cfg = CONFIGS[request.param]()
    ctx, G, H = build_pair(cfg)
    G.update_stencil()
    # operator-level parity shares the device's FP32 powf weights (checked on their own below)
    H.set_weights(G[0].getPenalty())
    H.update_stencil()
    yield cfg, ctx, G, H
    G.close()
    ctx.close()


def test_level_plan_and_activity_bit_exact(pair):
    cfg, ctx, G, H = pair
    assert G.n_grid() == H.nlev
    for i in range(H.nlev):
        L = H.levels[i]
        assert (G[i].nx, G[i].ny, G[i].nz, G[i].ratio) == (L.nx, L.ny, L.nz, L.ratio)
        assert np.array_equal(G[i].getVact(), H.arrs[i]["vact"])
        assert np.array_equal(G[i].getEact(), H.arrs[i]["eact"].ravel())


def test_penalty_weights_within_2ulp(pair):
    # powf(rho, p) in FP32 as the reference computes it; CUDA and glibc powf agree to ~1 ulp
    cfg, ctx, G, H = pair
    w = G[0].getPenalty()
    rho = cfg["rho"].ravel().astype(np.float32)
    ref = np.where(cfg["eact"].ravel() != 0, np.power(rho, np.float32(3.0)), np.float32(0)).astype(np.float32)
    ulp = np.spacing(np.maximum(np.abs(ref), np.finfo(np.float32).tiny))
    assert np.all(np.abs(w.astype(np.float64) - ref) <= 2 * ulp)


def test_template_matrix(pair):
    cfg, ctx, G, H = pair
    assert rel_err(G.template_matrix(), H.KE) < 1e-14


def test_surface_nodes_bit_exact(pair):
    cfg, ctx, G, H = pair
    assert np.array_equal(G.surface_nodes(), O.surface_nodes(cfg["eact"]).ravel())


def _rand_vec(G, i, seed):
    v = np.random.default_rng(seed).standard_normal(3 * G[i].nv)
    return v * np.tile(G[i].getVact(), 3)


def test_fine_residual_and_applyK(pair):
    cfg, ctx, G, H = pair
    u, f = _rand_vec(G, 0, 1), _rand_vec(G, 0, 2)
    G[0].setDisplacement(u)
    G[0].setForce(f)
    G[0].update_residual()
    r_gpu = G[0].getResidual()
    r_or = np.zeros_like(u)
    O.lib().or_fine_residual(H.lv(0), O.ptr(H.KE), O.ptr(u), O.ptr(f), O.ptr(r_or))
    assert rel_err(r_gpu, r_or) < FP64_TOL
    assert rel_err(G[0].applyK(u), H.applyK(u)) < FP64_TOL


@pytest.mark.parametrize("smoother", [rb.SMOOTH_GS, rb.SMOOTH_SGS, rb.SMOOTH_JACOBI])
def test_fine_smoothers(pair, smoother):
    cfg, ctx, G, H = pair
    u, f = _rand_vec(G, 0, 3), _rand_vec(G, 0, 4)
    G[0].setDisplacement(u)
    G[0].setForce(f)
    G[0].smooth(smoother, 2, 0.6)
    uo = u.copy()
    tmp = np.zeros_like(u)
    for s in range(2):
        if smoother == rb.SMOOTH_JACOBI:
            O.lib().or_fine_jacobi(H.lv(0), O.ptr(H.KE), O.ptr(uo), O.ptr(f), 0.6, O.ptr(tmp))
        else:
            O.lib().or_fine_gs(H.lv(0), O.ptr(H.KE), O.ptr(uo), O.ptr(f), 1 if smoother == rb.SMOOTH_SGS else 0)
    assert rel_err(G[0].getDisplacement(), uo) < 1e-10


@pytest.mark.parametrize("variant,ty,zc", [(0, 4, 8), (0, 2, 5), (0, 8, 3), (1, 2, 4), (1, 4, 16), (1, 8, 7),
                                           (1, 4, 1), (2, 2, 8), (2, 4, 3), (3, 4, 8), (3, 2, 5), (3, 8, 3),
                                           (3, 4, 1), (3, 2, 64), (5, 4, 8), (5, 8, 3), (5, 16, 1), (5, 4, 64),
                                           (5, 8, 5), (6, 4, 8), (6, 8, 3), (6, 4, 1), (6, 8, 64), (7, 4, 8),
                                           (7, 8, 3), (7, 4, 1), (7, 8, 64), (7, 6, 5), (7, 6, 32)])
def test_fine_kernel_variants(pair, variant, ty, zc):
    """Every launch shape of the finest-level kernels (shared-memory tile, register marching,
    register marching with prefetched output-stage loads, pipelined shared-memory tile,
    sum-factorised row marching, pipelined tile with TMA-staged node layers on 32- and 31-wide
    tiles where the node box's x extent is a multiple of 16) gives the oracle's residual, K u,
    Jacobi and Chebyshev results."""
    cfg, ctx, G, H = pair
    import ctypes as C

    for m in range(4):
        rb._capi.check(rb.lib().rt_set_tuning(G.handle, rb.FP64, m, variant, ty, zc), ctx.handle)
    u, f = _rand_vec(G, 0, 210), _rand_vec(G, 0, 211)
    G[0].setDisplacement(u)
    G[0].setForce(f)
    G[0].update_residual()
    r_or = np.zeros_like(u)
    O.lib().or_fine_residual(H.lv(0), O.ptr(H.KE), O.ptr(u), O.ptr(f), O.ptr(r_or))
    assert rel_err(G[0].getResidual(), r_or) < FP64_TOL
    assert rel_err(G[0].applyK(u), H.applyK(u)) < FP64_TOL
    G[0].smooth(rb.SMOOTH_JACOBI, 1, 0.6)
    uo, tmp = u.copy(), np.zeros_like(u)
    O.lib().or_fine_jacobi(H.lv(0), O.ptr(H.KE), O.ptr(uo), O.ptr(f), 0.6, O.ptr(tmp))
    assert rel_err(G[0].getDisplacement(), uo) < 1e-10
    H.set_lmax([G.smoother_lmax(i) for i in range(H.nlev - 1)])
    G[0].setDisplacement(u)
    G[0].smooth(rb.SMOOTH_CHEBY, 2)
    uo, un, d = u.copy(), np.zeros_like(u), np.zeros_like(u)
    for k in range(2):
        O.lib().or_fine_cheby(H.lv(0), O.ptr(H.KE), O.ptr(uo), O.ptr(f), O.ptr(un), O.ptr(d), k)
        uo, un = un, uo
    assert rel_err(G[0].getDisplacement(), uo) < 1e-9
    for m in range(4):  # back to the default shape
        rb._capi.check(rb.lib().rt_set_tuning(G.handle, rb.FP64, m, 1, 4, 16), ctx.handle)


FP32_TOL = 2e-6  # FP32 kernels against the FP64 oracle on random data (no cancellation)


@pytest.mark.parametrize("variant,ty,zc", [(0, 4, 8), (1, 2, 8), (2, 4, 8), (3, 4, 8), (3, 8, 3), (4, 4, 8),
                                           (4, 8, 16), (4, 2, 5), (4, 8, 1), (4, 4, 64), (5, 4, 8), (5, 8, 16),
                                           (5, 16, 3), (5, 8, 1), (5, 4, 64), (6, 4, 8), (6, 8, 16), (6, 4, 1),
                                           (6, 8, 64), (7, 4, 8), (7, 8, 16), (7, 4, 1), (7, 8, 64),
                                           (7, 6, 3), (7, 6, 32)])
def test_fp32_fine_kernels(pair, variant, ty, zc):
    """Every FP32 finest-level kernel variant (including the packed-pair tile kernel) gives the
    oracle's residual, K u, Jacobi and first Chebyshev step to FP32 accuracy."""
    cfg, ctx, G, H = pair
    for m in range(4):
        rb._capi.check(rb.lib().rt_set_tuning(G.handle, rb.FP32, m, variant, ty, zc), ctx.handle)
    u, f = _rand_vec(G, 0, 310), _rand_vec(G, 0, 311)
    G[0].setDisplacement(u)
    G[0].setForce(f)
    lib = rb.lib()
    rb._capi.check(lib.rt_fine_kernel_f32(G.handle, 0, 0.0), ctx.handle)
    r_or = np.zeros_like(u)
    O.lib().or_fine_residual(H.lv(0), O.ptr(H.KE), O.ptr(u), O.ptr(f), O.ptr(r_or))
    assert rel_err(G[0].getResidual(), r_or) < FP32_TOL
    rb._capi.check(lib.rt_fine_kernel_f32(G.handle, 1, 0.0), ctx.handle)
    assert rel_err(G[0].getResidual(), H.applyK(u)) < FP32_TOL
    rb._capi.check(lib.rt_fine_kernel_f32(G.handle, 2, 0.6), ctx.handle)
    uo, tmp = u.copy(), np.zeros_like(u)
    O.lib().or_fine_jacobi(H.lv(0), O.ptr(H.KE), O.ptr(uo), O.ptr(f), 0.6, O.ptr(tmp))
    assert rel_err(G[0].getResidual(), uo) < FP32_TOL
    H.set_lmax([G.smoother_lmax(i) for i in range(H.nlev - 1)])
    rb._capi.check(lib.rt_fine_kernel_f32(G.handle, 3, 0.0), ctx.handle)
    uc, un, d = u.copy(), np.zeros_like(u), np.zeros_like(u)
    O.lib().or_fine_cheby(H.lv(0), O.ptr(H.KE), O.ptr(uc), O.ptr(f), O.ptr(un), O.ptr(d), 0)
    assert rel_err(G[0].getResidual(), un) < FP32_TOL
    for m in range(4):
        rb._capi.check(rb.lib().rt_set_tuning(G.handle, rb.FP32, m, 1, 4, 16), ctx.handle)


@pytest.mark.parametrize("variant,ty,zc", [(0, 4, 8), (1, 2, 8), (2, 4, 8), (3, 4, 8), (3, 8, 2), (4, 8, 16),
                                           (4, 4, 8), (5, 8, 16), (5, 16, 32), (5, 4, 2), (6, 4, 8), (6, 8, 16),
                                           (7, 4, 8), (7, 8, 16), (7, 6, 16)])
def test_fp32_kernel_variants_in_pcg(pair, variant, ty, zc):
    """The FP32 finest-level kernels of every variant drive the mixed-precision PCG (FP32 Chebyshev
    V-cycles) to 1e-6 in the FP64 residual; FP32 rounding differs between variants, the iteration
    count stays within one step of the default shape's."""
    cfg, ctx, G, H = pair
    b = _rand_vec(G, 0, 81)
    if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF):
        b[np.tile(cfg["vfix"].ravel().astype(bool), 3)] = 0
    else:
        Ru = np.zeros(6 * b.size)
        O.lib().or_rigid_nodes(H.lv(0), O.ptr(Ru))
        O.lib().or_displacement_project(b.size // 3, O.ptr(Ru), O.ptr(b))
    params = G.params
    params.precision, params.smoother = rb.FP32, rb.SMOOTH_CHEBY
    params.pre_sweeps = params.post_sweeps = 4
    G.set_params(params)
    G.update_stencil()
    its = []
    for shape in ((1, 4, 16), (variant, ty, zc)):
        for m in range(4):
            rb._capi.check(rb.lib().rt_set_tuning(G.handle, rb.FP32, m, *shape), ctx.handle)
        G[0].setForce(b)
        G[0].reset_displacement()
        info = G.pcg(1e-6, 1000)
        assert info.status == 0 and info.rel_residual <= 1e-6
        r = (b - H.applyK(G[0].getDisplacement())) * np.tile(H.arrs[0]["vact"], 3)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.01e-6
        its.append(info.iterations)
    assert abs(its[1] - its[0]) <= 1, its
    for m in range(4):
        rb._capi.check(rb.lib().rt_set_tuning(G.handle, rb.FP32, m, 1, 4, 16), ctx.handle)
    params.precision, params.smoother = rb.FP64, rb.SMOOTH_SGS
    params.pre_sweeps = params.post_sweeps = 1
    G.set_params(params)
    G.update_stencil()


@pytest.mark.parametrize("bf16,variant", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_level_kernel_variants_in_pcg(pair, bf16, variant):
    """Both stencil-level kernels of the FP32 smoother (lane-split, bulk-copy), on the FP32 and the
    BF16 stencil copies, drive the mixed-precision PCG to 1e-6 in the FP64 residual."""
    cfg, ctx, G, H = pair
    b = _rand_vec(G, 0, 82)
    if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF):
        b[np.tile(cfg["vfix"].ravel().astype(bool), 3)] = 0
    else:
        Ru = np.zeros(6 * b.size)
        O.lib().or_rigid_nodes(H.lv(0), O.ptr(Ru))
        O.lib().or_displacement_project(b.size // 3, O.ptr(Ru), O.ptr(b))
    params = G.params
    params.precision, params.smoother = rb.FP32, rb.SMOOTH_CHEBY
    params.pre_sweeps = params.post_sweeps = 4
    params.coarse_bf16 = bf16
    G.set_params(params)
    G.update_stencil()
    rb._capi.check(rb.lib().rt_set_level_kernel(G.handle, bf16, variant), ctx.handle)
    G[0].setForce(b)
    G[0].reset_displacement()
    info = G.pcg(1e-6, 1000)
    assert info.status == 0 and info.rel_residual <= 1e-6
    r = (b - H.applyK(G[0].getDisplacement())) * np.tile(H.arrs[0]["vact"], 3)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.01e-6
    rb._capi.check(rb.lib().rt_set_level_kernel(G.handle, 0, 0), ctx.handle)
    rb._capi.check(rb.lib().rt_set_level_kernel(G.handle, 1, 1), ctx.handle)
    params.precision, params.smoother = rb.FP64, rb.SMOOTH_SGS
    params.pre_sweeps = params.post_sweeps = 1
    params.coarse_bf16 = 0
    G.set_params(params)
    G.update_stencil()


def test_autotune_keeps_results(pair):
    cfg, ctx, G, H = pair
    shapes = G.autotune(reps=2)
    assert set(shapes) >= {"residual_f32", "chebyshev_f64"}
    u, f = _rand_vec(G, 0, 220), _rand_vec(G, 0, 221)
    G[0].setDisplacement(u)
    G[0].setForce(f)
    G[0].update_residual()
    r_or = np.zeros_like(u)
    O.lib().or_fine_residual(H.lv(0), O.ptr(H.KE), O.ptr(u), O.ptr(f), O.ptr(r_or))
    assert rel_err(G[0].getResidual(), r_or) < FP64_TOL


def test_galerkin_stencils(pair):
    cfg, ctx, G, H = pair
    for i in range(1, H.nlev):
        assert rel_err(G[i].getStencil(), H.arrs[i]["st"]) < FP64_TOL, f"level {i}"


def test_transfers(pair):
    cfg, ctx, G, H = pair
    for i in range(1, H.nlev):
        rf = _rand_vec(G, i - 1, 10 + i)
        G[i - 1].setResidual(rf)
        G[i].restrict_residual()
        fc = np.zeros(3 * G[i].nv)
        O.lib().or_restrict(H.lv(i - 1), H.lv(i), O.ptr(rf), O.ptr(fc))
        assert rel_err(G[i].getForce(), fc) < 1e-13
        uc = _rand_vec(G, i, 20 + i)
        uf = _rand_vec(G, i - 1, 30 + i)
        G[i].setDisplacement(uc)
        G[i - 1].setDisplacement(uf)
        G[i - 1].prolongate_correction()
        uf2 = uf.copy()
        O.lib().or_prolong_add(H.lv(i - 1), H.lv(i), O.ptr(uc), O.ptr(uf2))
        assert rel_err(G[i - 1].getDisplacement(), uf2) < 1e-13


def test_coarse_level_ops(pair):
    cfg, ctx, G, H = pair
    for i in range(1, H.nlev):
        u, f = _rand_vec(G, i, 40 + i), _rand_vec(G, i, 50 + i)
        G[i].setDisplacement(u)
        G[i].setForce(f)
        G[i].update_residual()
        r = np.zeros_like(u)
        O.lib().or_st_residual(H.lv(i), O.ptr(u), O.ptr(f), O.ptr(r))
        assert rel_err(G[i].getResidual(), r) < FP64_TOL
        G[i].gs_relax(1)
        uo = u.copy()
        O.lib().or_st_gs(H.lv(i), O.ptr(uo), O.ptr(f), 0)
        # the block division amplifies FP64 rounding on the 1e9-contrast stencils
        assert rel_err(G[i].getDisplacement(), uo) < 1e-9


def test_chebyshev_bounds_and_steps(pair):
    cfg, ctx, G, H = pair
    lm = [G.smoother_lmax(i) for i in range(H.nlev - 1)]
    # device power iteration vs the oracle's own estimate (different rounding, same start vector)
    for i in range(H.nlev - 1):
        assert abs(lm[i] - H.LA[i].lmax) <= 1e-6 * H.LA[i].lmax
    H.set_lmax(lm)
    for i in range(H.nlev - 1):
        u, f = _rand_vec(G, i, 110 + i), _rand_vec(G, i, 120 + i)
        G[i].setDisplacement(u)
        G[i].setForce(f)
        G[i].smooth(rb.SMOOTH_CHEBY, 3)
        uo, un = u.copy(), np.zeros_like(u)
        d = np.zeros_like(u)
        for k in range(3):
            if i == 0:
                O.lib().or_fine_cheby(H.lv(0), O.ptr(H.KE), O.ptr(uo), O.ptr(f), O.ptr(un), O.ptr(d), k)
            else:
                O.lib().or_st_cheby(H.lv(i), O.ptr(uo), O.ptr(f), O.ptr(un), O.ptr(d), k)
            uo, un = un, uo
        assert rel_err(G[i].getDisplacement(), uo) < 1e-9, f"level {i}"


@pytest.mark.parametrize("nsteps,form", [(3, 1), (8, 1), (3, 2), (8, 2)])
def test_fused_chebyshev_sweeps(pair, nsteps, form):
    """FP32 Chebyshev smoothing of every stencil level as one cooperative launch (grid barrier
    between the steps), in the resident (form 1 on these small levels) and the streaming form
    (2), gives the separate launches' result, and both follow the oracle's FP64 steps to FP32
    accuracy; odd step counts end with the copy back into u."""
    cfg, ctx, G, H = pair
    lm = [G.smoother_lmax(i) for i in range(H.nlev - 1)]
    H.set_lmax(lm)
    lib = rb.lib()
    rb._capi.check(lib.rt_set_level_kernel(G.handle, 0, 0), ctx.handle)  # lane-split: same sums as fused
    for i in range(1, H.nlev - 1):
        u, f = _rand_vec(G, i, 130 + i), _rand_vec(G, i, 140 + i)
        out = []
        for fused in (0, form):
            rb._capi.check(lib.rt_set_level_fused(G.handle, i, fused), ctx.handle)
            G[i].setDisplacement(u)
            G[i].setForce(f)
            rb._capi.check(lib.rt_smooth_f32(G.handle, i, rb.SMOOTH_CHEBY, nsteps, 0.0), ctx.handle)
            out.append(G[i].getDisplacement())
        rb._capi.check(lib.rt_set_level_fused(G.handle, i, 0), ctx.handle)
        assert rel_err(out[1], out[0]) < 1e-6, f"level {i}"
        uo, un, d = u.copy(), np.zeros_like(u), np.zeros_like(u)
        for k in range(nsteps):
            O.lib().or_st_cheby(H.lv(i), O.ptr(uo), O.ptr(f), O.ptr(un), O.ptr(d), k)
            uo, un = un, uo
        assert rel_err(out[1], uo) < 1e-3, f"level {i}"


def test_fused_chebyshev_in_pcg(pair):
    """The mixed-precision PCG with every stencil level's Chebyshev sweeps fused reaches 1e-6 in the
    FP64 residual within one iteration of the separate launches' count."""
    cfg, ctx, G, H = pair
    b = _rand_vec(G, 0, 86)
    if cfg["mode"] not in (rb.MODE_WSCF, rb.MODE_WSFF):
        return  # the rigid-mode projection is covered by the other PCG tests
    b[np.tile(cfg["vfix"].ravel().astype(bool), 3)] = 0
    params = G.params
    params.precision, params.smoother = rb.FP32, rb.SMOOTH_CHEBY
    params.pre_sweeps = params.post_sweeps = 2
    params.coarse_sweeps = 8
    G.set_params(params)
    G.update_stencil()
    its = []
    for fused in (0, 1):
        for i in range(1, G.n_grid() - 1):
            rb._capi.check(rb.lib().rt_set_level_fused(G.handle, i, fused), ctx.handle)
        G[0].setForce(b)
        G[0].reset_displacement()
        info = G.pcg(1e-6, 1000)
        assert info.status == 0 and info.rel_residual <= 1e-6
        r = (b - H.applyK(G[0].getDisplacement())) * np.tile(H.arrs[0]["vact"], 3)
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.01e-6
        its.append(info.iterations)
    assert abs(its[1] - its[0]) <= 1
    for i in range(1, G.n_grid() - 1):
        rb._capi.check(rb.lib().rt_set_level_fused(G.handle, i, 0), ctx.handle)
    params.precision, params.smoother = rb.FP64, rb.SMOOTH_SGS
    params.pre_sweeps = params.post_sweeps = 1
    params.coarse_sweeps = 0
    G.set_params(params)
    G.update_stencil()


def test_coarsest_solve(pair):
    cfg, ctx, G, H = pair
    last = H.nlev - 1
    f = _rand_vec(G, last, 60)
    G[last].setForce(f)
    G[last].solve_fem_host()
    H.arrs[last]["f"][:] = f
    O.lib().or_coarsest_solve(H.lv(last))
    assert rel_err(G[last].getDisplacement(), H.arrs[last]["u"]) < 1e-7


def test_vcycle_sequence(pair):
    cfg, ctx, G, H = pair
    f = _rand_vec(G, 0, 70)
    G[0].setForce(f)
    G[0].reset_displacement()
    H.arrs[0]["f"][:] = f
    H.arrs[0]["u"][:] = 0
    for it in range(4):
        rg = G.v_cycle(1, 1)
        ro = H.vcycle(O.SMOOTH_GS, 1, 1)
        assert abs(rg - ro) <= 1e-7 * ro, (it, rg, ro)
    assert rel_err(G[0].getDisplacement(), H.arrs[0]["u"]) < 1e-8


@pytest.mark.parametrize("precision,smoother,sweeps,bf16", [(rb.FP64, rb.SMOOTH_SGS, 1, 0),
                                                            (rb.FP32, rb.SMOOTH_SGS, 1, 0),
                                                            (rb.FP32, rb.SMOOTH_CHEBY, 4, 0),
                                                            (rb.FP32, rb.SMOOTH_CHEBY, 4, 1),
                                                            (rb.FP32, rb.SMOOTH_JACOBI, 2, 1),
                                                            (rb.FP64, rb.SMOOTH_JACOBI, 2, 0),
                                                            (rb.FP64_FINE, rb.SMOOTH_CHEBY, 4, 0),
                                                            (rb.FP64_FINE, rb.SMOOTH_SGS, 1, 0)])
def test_pcg_to_1e6(pair, precision, smoother, sweeps, bf16):
    """MG-PCG to 1e-6 in every precision form; bf16=1 smooths levels >= 1 with BF16-stored stencils,
    which changes the preconditioner only: the FP64 residual of the answer still meets the tolerance."""
    cfg, ctx, G, H = pair
    b = _rand_vec(G, 0, 80)
    if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF):
        b[np.tile(cfg["vfix"].ravel().astype(bool), 3)] = 0
    else:
        # without supports the load must be self-equilibrated: remove rigid components
        Ru = np.zeros(6 * b.size)
        O.lib().or_rigid_nodes(H.lv(0), O.ptr(Ru))
        O.lib().or_displacement_project(b.size // 3, O.ptr(Ru), O.ptr(b))
    params = G.params
    params.precision = precision
    params.smoother = smoother
    params.pre_sweeps = params.post_sweeps = sweeps
    params.jacobi_omega = 0.5
    params.coarse_bf16 = bf16
    G.set_params(params)
    G.update_stencil()
    G[0].setForce(b)
    G[0].reset_displacement()
    if bf16:
        ctx.profile(True)
        ctx.profile_reset()
    info = G.pcg(1e-6, 1000)
    if bf16:
        st = ctx.profile_stats()
        ctx.profile(False)
        if G.n_grid() > 2:  # a smoothed coarse level exists: its smoother read the BF16 stencils
            assert sum(v[0] for k, v in st.items() if k.startswith("st_") and "_bf16" in k) > 0, st
        assert not any(k.startswith("st_") and "_f32" in k and "residual" not in k for k in st), st
    assert info.status == 0 and info.rel_residual <= 1e-6
    x = G[0].getDisplacement()
    # FP64 residual check of the returned solution with the oracle operator
    r = b - H.applyK(x)
    r *= np.tile(H.arrs[0]["vact"], 3)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.01e-6
    xo, ito, rro = H.pcg(b, tol=1e-6, smoother=O.SMOOTH_SGS)
    assert abs(b @ x - b @ xo) <= 1e-5 * abs(b @ xo)
    params.precision = rb.FP64
    params.smoother = rb.SMOOTH_SGS
    params.pre_sweeps = params.post_sweeps = 1
    params.coarse_bf16 = 0
    G.set_params(params)
    G.update_stencil()


@pytest.mark.parametrize("gamma", [1, 2])
def test_pcg_fp32_krylov_refinement(pair, gamma):
    """FP32 Krylov vectors with FP64 iterative refinement (krylov_fp32): the answer meets 1e-6
    in the FP64 residual computed by the oracle's operator; modes without supports take the
    FP64-vector form."""
    cfg, ctx, G, H = pair
    b = _rand_vec(G, 0, 83)
    if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF):
        b[np.tile(cfg["vfix"].ravel().astype(bool), 3)] = 0
    else:
        Ru = np.zeros(6 * b.size)
        O.lib().or_rigid_nodes(H.lv(0), O.ptr(Ru))
        O.lib().or_displacement_project(b.size // 3, O.ptr(Ru), O.ptr(b))
    params = G.params
    params.precision, params.smoother = rb.FP32, rb.SMOOTH_CHEBY
    params.pre_sweeps = params.post_sweeps = 2
    params.cycle_gamma, params.krylov_fp32 = gamma, 1
    G.set_params(params)
    G.update_stencil()
    G[0].setForce(b)
    G[0].reset_displacement()
    info = G.pcg(1e-6, 1000)
    assert info.status == 0 and info.rel_residual <= 1e-6
    r = (b - H.applyK(G[0].getDisplacement())) * np.tile(H.arrs[0]["vact"], 3)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1.01e-6
    params.precision, params.smoother = rb.FP64, rb.SMOOTH_SGS
    params.pre_sweeps = params.post_sweeps = 1
    params.cycle_gamma, params.krylov_fp32 = 1, 0
    G.set_params(params)
    G.update_stencil()


@pytest.mark.parametrize("krylov", [0, 2])
def test_graph_launch_accounting(pair, krylov):
    """A captured PCG loop adds its kernels to the launch count once per executed iteration:
    the count equals that of the same solve run uncaptured, one launch per kernel (profiling
    mode), with the same iteration count."""
    cfg, ctx, G, H = pair
    b = _rand_vec(G, 0, 85)
    if cfg["mode"] not in (rb.MODE_WSCF, rb.MODE_WSFF):
        return  # the projection of rigid modes is covered above; the accounting is mode independent
    b[np.tile(cfg["vfix"].ravel().astype(bool), 3)] = 0
    params = G.params
    params.precision, params.smoother, params.krylov_fp32 = rb.FP32, rb.SMOOTH_CHEBY, krylov
    G.set_params(params)
    G.update_stencil()
    runs = []
    for prof in (False, True):
        ctx.profile(prof)
        G[0].setForce(b)
        G[0].reset_displacement()
        l0 = ctx.launches()
        info = G.pcg(1e-6, 1000)
        runs.append((ctx.launches() - l0, info.iterations, info.status))
    ctx.profile(False)
    assert runs[0] == runs[1] and runs[0][2] == 0 and runs[0][0] > 10 * runs[0][1]
    params.precision, params.smoother, params.krylov_fp32 = rb.FP64, rb.SMOOTH_SGS, 0
    G.set_params(params)
    G.update_stencil()


def test_modified_pm_parity(pair):
    cfg, ctx, G, H = pair
    lam, info = G.worst_case(rb.WORST_MODPM, 500, 0.0, seed=9)
    nl = cfg["load_nodes"].size
    fs = np.zeros(3 * nl)
    it = np.zeros(1, np.int32)
    constrain = 1 if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_NSCF) else 0
    ws = cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF)
    pos = np.stack(np.unravel_index(cfg["load_nodes"], cfg["vfix"].shape)[::-1], 1).astype(np.float64)
    Rd = np.zeros(6 * 3 * nl)
    nrig = 0 if ws else O.lib().or_rigid_basis(nl, O.ptr(np.ascontiguousarray(pos)),
                                                O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), constrain,
                                                O.ptr(Rd))
    Ru = None
    if not ws:
        Ru = np.zeros(6 * 3 * (H.arrs[0]["u"].size // 3))
        O.lib().or_rigid_nodes(H.lv(0), O.ptr(Ru))
    lam_o = O.lib().or_modified_pm(H.LA, H.nlev, O.ptr(H.KE), nl, O.ptr(cfg["load_nodes"]),
                                   O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), constrain, nrig,
                                   O.ptr(Rd) if nrig else None, O.ptr(Ru) if Ru is not None else None, 9, 500,
                                   O.ptr(it), O.ptr(fs))
    assert info.iterations == it[0] or abs(info.iterations - it[0]) <= 1
    assert abs(lam - lam_o) <= 1e-6 * abs(lam_o)


def test_lanczos_parity(pair):
    cfg, ctx, G, H = pair
    params = G.params
    lam, info = G.worst_case(rb.WORST_LANCZOS, 16, 1e-10, seed=13)
    nl = cfg["load_nodes"].size
    nv = H.arrs[0]["u"].size // 3
    constrain = 1 if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_NSCF) else 0
    ws = cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF)
    pos = np.stack(np.unravel_index(cfg["load_nodes"], cfg["vfix"].shape)[::-1], 1).astype(np.float64)
    Rd = np.zeros(6 * 3 * nl)
    nrig = 0 if ws else O.lib().or_rigid_basis(nl, O.ptr(np.ascontiguousarray(pos)),
                                                O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), constrain,
                                                O.ptr(Rd))
    k = 16
    work = np.zeros((k + 1) * 3 * nl + 10 * 3 * nv)
    lo = np.zeros(1)
    O.lib().or_lanczos(H.LA, H.nlev, O.ptr(H.KE), O.SMOOTH_SGS, 1, 1, 0.6, nl, O.ptr(cfg["load_nodes"]),
                       O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), constrain, nrig,
                       O.ptr(Rd) if nrig else None, 13, k, 1e-10, 500, O.ptr(lo), None, O.ptr(work))
    assert abs(lam - lo[0]) <= 1e-7 * abs(lo[0])
    # the returned load/displacement realise the eigenvalue: f.u = lambda with ||f|| = 1
    f = G[0].getForce()
    u = G[0].getDisplacement()
    assert abs(np.linalg.norm(f) - 1) < 1e-9
    assert abs(f @ u - lam) <= 1e-6 * lam


def test_sensitivity_filter_oc(pair):
    cfg, ctx, G, H = pair
    u = _rand_vec(G, 0, 90) * 1e-3
    G[0].setDisplacement(u)
    import ctypes as C

    rb.lib().rt_sensitivity(G.handle, 0)
    s_gpu = G[0].getSens()
    nz, ny, nx = cfg["eact"].shape
    s_or = np.zeros(nx * ny * nz, np.float32)
    rho = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
    O.lib().or_sensitivity(nx, ny, nz, O.ptr(H.arrs[0]["eact"]), O.ptr(rho), 3.0, O.ptr(H.KE), O.ptr(u), O.ptr(s_or))
    assert rel_err(s_gpu, s_or) < 1e-6
    # filter from the same input
    G[0].setSens(s_or)
    G[0].filterSensitivity(2.0)
    f_or = np.zeros_like(s_or)
    O.lib().or_filter(nx, ny, nz, O.ptr(H.arrs[0]["eact"]), 2.0, O.ptr(s_or), O.ptr(f_or))
    assert rel_err(G[0].getSens(), f_or) < 1e-6
    # OC update from the same sensitivities
    G[0].setSens(f_or)
    G[0].setRho(rho)
    lam = C.c_float()
    trials = C.c_int()
    rb._capi.check(rb.lib().rt_oc_update(G.handle, 0.4, C.byref(lam), C.byref(trials)), ctx.handle)
    rho_o = rho.copy()
    tmp = np.zeros_like(rho_o)
    it = np.zeros(1, np.int32)
    lam_o = O.lib().or_oc_update(rho_o.size, O.ptr(H.arrs[0]["eact"]), None, O.ptr(rho_o), O.ptr(f_or), 0.4, 0.03,
                                 0.5, 1e-3, int(H.arrs[0]["eact"].sum()), O.ptr(it), O.ptr(tmp))
    assert np.abs(G[0].getRho() - rho_o).max() <= 1e-4
    assert abs(lam.value - lam_o) <= 1e-3 * abs(lam_o)
    # with shell elements (held at 1): the same update with the oracle's shell mask
    shell = (np.random.default_rng(7).random(rho.size) < 0.2).astype(np.uint8) & H.arrs[0]["eact"].ravel()
    G.set_shell(shell)
    G[0].setSens(f_or)
    G[0].setRho(rho)
    rb._capi.check(rb.lib().rt_oc_update(G.handle, 0.4, C.byref(lam), C.byref(trials)), ctx.handle)
    rho_s = rho.copy()
    lam_s = O.lib().or_oc_update(rho_s.size, O.ptr(H.arrs[0]["eact"]), O.ptr(shell), O.ptr(rho_s), O.ptr(f_or), 0.4,
                                 0.03, 0.5, 1e-3, int(H.arrs[0]["eact"].sum()), O.ptr(it), O.ptr(tmp))
    got = G[0].getRho()
    assert np.all(got[shell.astype(bool)] == 1.0)
    assert np.abs(got - rho_s).max() <= 1e-4
    assert abs(lam.value - lam_s) <= 1e-3 * abs(lam_s)
    G.set_shell(None)
    G[0].setRho(rho)
    G.update_stencil()


def test_ref_gs_layout(pair):
    cfg, ctx, G, H = pair
    vm, ngs, gsn = G[0].ref_gs_map()
    act = G[0].getVact().astype(bool)
    assert np.all(vm[~act] == -1) and np.all(vm[act] >= 0)
    assert ngs == gsn.sum() and all(g % 32 == 0 for g in gsn)
    # within a colour, slots follow the dense (bit) order, as enumerate_gs_subset does
    u = _rand_vec(G, 0, 100)
    G[0].setDisplacement(u)
    ref = G[0].getDisplacement(rb.LAYOUT_REF_GS)
    nv = G[0].nv
    for c in range(3):
        assert np.array_equal(ref[c * ngs + vm[act]], u[c * nv + np.flatnonzero(act)])
    G[0].setDisplacement(np.zeros_like(u))
    G[0].setDisplacement(ref, rb.LAYOUT_REF_GS)
    assert np.array_equal(G[0].getDisplacement(), u)


def test_cube_bits_bit_exact():
    import ctypes as C

    ctx = rb.Context(0)
    rng = np.random.default_rng(21)
    R = 40
    dense = (rng.random((R, R, R)) < 0.35).astype(np.uint8)
    bits = np.packbits(dense.ravel(), bitorder="little").view(np.uint32).copy()
    bits = np.concatenate([bits, np.zeros(((R ** 3 + 31) // 32) - bits.size, np.uint32)])
    vb = np.zeros(((R + 1) ** 3 + 31) // 32, np.uint32)
    rb._capi.check(rb.lib().rt_cube_vertex_bits(ctx.handle, R, bits.ctypes.data, vb.ctypes.data), ctx.handle)
    assert np.array_equal(vb, O.cube_vbits(R, bits))
    ec = np.zeros(((R // 2) ** 3 + 31) // 32, np.uint32)
    rb._capi.check(rb.lib().rt_cube_coarsen_bits(ctx.handle, R, bits.ctypes.data, ec.ctypes.data), ctx.handle)
    assert np.array_equal(ec, O.cube_coarsen(R, bits))
    ctx.close()


def test_gen_from_mesh_bits_equals_box():
    # genFromMesh(solid_bit, reso) and the dense-box builder give the same hierarchy
    cfg = CONFIGS["ragged_arch"]()
    nz, ny, nx = cfg["eact"].shape
    R = 32
    cube = np.zeros((R, R, R), np.uint8)
    cube[:nz, :ny, :nx] = cfg["eact"]
    bits = np.packbits(cube.ravel(), bitorder="little").view(np.uint32).copy()
    ctx = rb.Context(0)
    G1 = rb.HierarchyGrid(ctx, rb.default_params())
    G1.genFromMesh(bits, [R, R, R])
    G2 = rb.HierarchyGrid(ctx, rb.default_params())
    G2.genFromBox(cfg["eact"])
    assert G1.n_grid() == G2.n_grid()
    for i in range(G1.n_grid()):
        assert (G1[i].nx, G1[i].ny, G1[i].nz) == (G2[i].nx, G2[i].ny, G2[i].nz)
        assert np.array_equal(G1[i].getEact(), G2[i].getEact())
    G1.close()
    G2.close()
    ctx.close()


def test_errors_are_reported_not_fatal():
    ctx = rb.Context(0)
    G = rb.HierarchyGrid(ctx, rb.default_params())
    with pytest.raises(rb.RTError):
        G.genFromBox(np.ones((4, 4, 4), np.uint8))  # too small for a hierarchy
    G.genFromBox(np.ones((8, 8, 12), np.uint8))
    with pytest.raises(rb.RTError):
        G.v_cycle()  # stencil not assembled yet
    with pytest.raises(rb.RTError):
        G.set_load_nodes(np.array([10 ** 9]), np.zeros((1, 3)))
    G.close()
    ctx.close()
