"""Solve workspaces, batched MG-PCG in one CUDA graph launch, and block Lanczos (GPU).

The batched path must reproduce the single-solve path bit for bit (same kernels, same
launch shapes, fixed-order reductions), and block Lanczos must reach the same largest
eigenvalue of the load-space compliance operator as the oracle's Lanczos restatement
(the worst-case load problem of optimization/optimization.cpp:123-261).
"""
import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from gpu_common import CONFIGS, E, NU, P, build_pair

pytestmark = pytest.mark.gpu


def _params(cfg, precision=rb.FP64, smoother=rb.SMOOTH_SGS, sweeps=1):
    return rb.default_params(mode=cfg["mode"], youngs_modulus=E, poisson_ratio=NU, power_penalty=P, min_rho=1e-3,
                             precision=precision, smoother=smoother, pre_sweeps=sweeps, post_sweeps=sweeps)


def _grid(ctx, cfg, params):
    G = rb.HierarchyGrid(ctx, params)
    G.genFromBox(cfg["eact"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    if cfg["load_nodes"] is not None and len(cfg["load_nodes"]):
        G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    G.update_stencil()
    return G


def _rhs(G, cfg, seed):
    vact = G[0].getVact().astype(np.float64)
    free = vact * (1.0 - cfg["vfix"].ravel().astype(np.float64))
    f = np.random.default_rng(seed).standard_normal(3 * G[0].nv) * np.tile(free, 3)
    if cfg["mode"] in (rb.MODE_NSCF, rb.MODE_NSFF):
        return None  # no-support instances need an admissible load; the fixture configs below have supports
    return f


def test_workspace_matches_parent():
    cfg = CONFIGS["worstcase"]()
    ctx = rb.Context(0)
    G = _grid(ctx, cfg, _params(cfg))
    f = _rhs(G, cfg, 1)
    G[0].setForce(f)
    G[0].setDisplacement(np.zeros_like(f))
    info = G.pcg(1e-8, 500)
    u_parent = G[0].getDisplacement()
    W = G.workspace()
    W[0].setForce(f)
    W[0].setDisplacement(np.zeros_like(f))
    info_w = W.pcg(1e-8, 500)
    assert info.status == rb._capi.RT_OK and info_w.status == rb._capi.RT_OK
    assert info_w.iterations == info.iterations
    assert np.array_equal(W[0].getDisplacement(), u_parent)
    # the workspace shares the operator: it refuses calls that would change it
    for call in (lambda: W.set_support(cfg["vfix"]), lambda: W.update_stencil(), lambda: W[0].setRho(cfg["rho"].ravel()),
                 lambda: W.worst_case(rb.WORST_LANCZOS, 4, 1e-6)):
        with pytest.raises(rb.RTError) as e:
            call()
        assert e.value.status == rb._capi.RT_ESTATE
    # a density change on the parent reaches the workspace after the parent's update_stencil
    G[0].setRho(np.clip(cfg["rho"].ravel() * 0.9, 1e-3, 1.0))
    G.update_stencil()
    G[0].setDisplacement(np.zeros_like(f))
    info2 = G.pcg(1e-8, 500)
    W[0].setDisplacement(np.zeros_like(f))
    info2_w = W.pcg(1e-8, 500)
    assert info2_w.iterations == info2.iterations
    assert np.array_equal(W[0].getDisplacement(), G[0].getDisplacement())
    G.close()
    ctx.close()


@pytest.mark.parametrize("form", ["fp64_sgs", "fp32_cheby"])
def test_pcg_batch_matches_single(form):
    prec, sm, sw = (rb.FP64, rb.SMOOTH_SGS, 1) if form == "fp64_sgs" else (rb.FP32, rb.SMOOTH_CHEBY, 4)
    ctx = rb.Context(0)
    cfgs = [CONFIGS["cantilever"](), CONFIGS["worstcase"](), CONFIGS["ragged_arch"]()]
    grids = [_grid(ctx, c, _params(c, prec, sm, sw)) for c in cfgs]
    # two extra right-hand sides on the second instance's operator
    insts = grids + [grids[1].workspace(), grids[1].workspace()]
    inst_cfg = cfgs + [cfgs[1], cfgs[1]]
    rhs = [_rhs(g, c, 10 + i) for i, (g, c) in enumerate(zip(insts, inst_cfg))]
    single = []
    for g, f in zip(insts, rhs):
        g[0].setForce(f)
        g[0].setDisplacement(np.zeros_like(f))
        info = g.pcg(1e-7, 500)
        single.append((info.iterations, g[0].getDisplacement()))
        g[0].setDisplacement(np.zeros_like(f))
    for rep in range(2):  # the second launch reuses the cached graph
        infos = rb.pcg_batch(insts, 1e-7, 500)
        for (it, u), info, g in zip(single, infos, insts):
            assert info.status == rb._capi.RT_OK
            assert info.iterations == it
            assert np.array_equal(g[0].getDisplacement(), u)
            g[0].setDisplacement(np.zeros_like(u))
    for g in grids:
        g.close()
    ctx.close()


def test_pcg_batch_rejects_bad_input():
    cfg = CONFIGS["worstcase"]()
    ctx = rb.Context(0)
    G = _grid(ctx, cfg, _params(cfg))
    with pytest.raises(rb.RTError):
        rb.pcg_batch([G, G], 1e-6, 10)
    ctx2 = rb.Context(0)
    G2 = _grid(ctx2, cfg, _params(cfg))
    with pytest.raises(rb.RTError):
        rb.pcg_batch([G, G2], 1e-6, 10)
    G.close()
    G2.close()
    ctx.close()
    ctx2.close()


@pytest.mark.parametrize("name", ["worstcase", "free_nscf"])
def test_block_lanczos_parity(name):
    cfg = CONFIGS[name]()
    ctx, G, H = build_pair(cfg)
    G.update_stencil()
    lam_b, info_b = G.worst_case_block(block_size=4, n_blocks=8, inner_tol=1e-10, seed=21)
    # the oracle's Lanczos restatement, run to a Krylov dimension where the top eigenvalue has converged
    nl = cfg["load_nodes"].size
    nv = H.arrs[0]["u"].size // 3
    constrain = 1 if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_NSCF) else 0
    ws = cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF)
    pos = np.stack(np.unravel_index(cfg["load_nodes"], cfg["vfix"].shape)[::-1], 1).astype(np.float64)
    Rd = np.zeros(6 * 3 * nl)
    nrig = 0 if ws else O.lib().or_rigid_basis(nl, O.ptr(np.ascontiguousarray(pos)),
                                                O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), constrain,
                                                O.ptr(Rd))
    k = 40
    work = np.zeros((k + 1) * 3 * nl + 10 * 3 * nv)
    lo = np.zeros(1)
    O.lib().or_lanczos(H.LA, H.nlev, O.ptr(H.KE), O.SMOOTH_SGS, 1, 1, 0.6, nl, O.ptr(cfg["load_nodes"]),
                       O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), constrain, nrig,
                       O.ptr(Rd) if nrig else None, 13, k, 1e-10, 500, O.ptr(lo), None, O.ptr(work))
    assert abs(lam_b - lo[0]) <= 1e-6 * abs(lo[0])
    assert info_b.iterations >= 1 and info_b.inner_iterations > 0
    # the returned load/displacement realise the eigenvalue: f.u = lambda with ||f|| = 1
    f = G[0].getForce()
    u = G[0].getDisplacement()
    assert abs(np.linalg.norm(f) - 1) < 1e-9
    assert abs(f @ u - lam_b) <= 1e-6 * lam_b
    # the rt_worst_case entry (block size 8, Krylov dimension rounded up to a multiple of 8): 8 block
    # steps, so that the block Krylov polynomial has the degree of the 4 x 8 call above
    lam_w, _ = G.worst_case(rb.WORST_BLOCK_LANCZOS, 64, 1e-10, seed=21)
    assert abs(lam_w - lo[0]) <= 1e-6 * abs(lo[0])
    G.close()
    ctx.close()


def test_context_outlives_its_hierarchies():
    # destroying the context first (as a garbage collector may) leaves its hierarchies usable
    cfg = CONFIGS["worstcase"]()
    ctx = rb.Context(0)
    G = _grid(ctx, cfg, _params(cfg))
    W = G.workspace()
    rb.lib().rt_ctx_destroy(ctx.handle)
    ctx._h = type(ctx._h)()  # the Python wrapper no longer owns the handle
    f = _rhs(G, cfg, 3)
    W[0].setForce(f)
    W[0].setDisplacement(np.zeros_like(f))
    assert W.pcg(1e-6, 500).status == rb._capi.RT_OK
    W.close()
    G.close()


def test_precision_fallback_at_scale():
    """On the 256x256x128 smoothed-random box (stiffness contrast 1e9) FP32 V-cycles stop reducing
    the residual; the solve continues from its iterate with FP64 V-cycles and reaches 1e-6."""
    from robtop_b200 import configs

    cfg = configs.worst_case_box(256, 256, 128, seed=0)
    ctx = rb.Context(0)
    G = _grid(ctx, cfg, _params(cfg, rb.FP32, rb.SMOOTH_CHEBY, 4))
    f = np.zeros(3 * G[0].nv)
    rng = np.random.default_rng(5)
    for c in range(3):
        f[c * G[0].nv + cfg["load_nodes"]] = rng.standard_normal(cfg["load_nodes"].size)
    G[0].setForce(f)
    G[0].setDisplacement(np.zeros_like(f))
    assert rb.lib().rt_hier_precision_fallbacks(G.handle) == 0
    info = G.pcg(1e-6, 3000)
    assert info.status == rb._capi.RT_OK and info.rel_residual <= 1e-6
    assert rb.lib().rt_hier_precision_fallbacks(G.handle) == 1
    G.close()
    ctx.close()
