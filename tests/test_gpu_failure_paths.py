"""Failure detection without a GPU fault: a bounded device wait that runs out, and non-finite
data injected from the host.  Every case must end in an error status the host reads, with the
context still usable afterwards."""
import ctypes as C

import numpy as np
import pytest

import robtop_b200 as rb
from robtop_b200 import configs

pytestmark = pytest.mark.gpu


def _grid(ctx, cfg):
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0, min_rho=1e-3,
                          precision=rb.FP32, smoother=rb.SMOOTH_CHEBY, pre_sweeps=2, post_sweeps=2, coarse_sweeps=4)
    G = rb.HierarchyGrid(ctx, p)
    G.genFromBox(cfg["eact"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    G.update_stencil()
    return G


def test_grid_barrier_wait_runs_out_and_context_recovers():
    """The fused Chebyshev sweep's grid barrier with a wait limit of zero polls: the blocks that
    are not last give up at once, the solve reports the barrier and returns; with the default
    limit the same hierarchy then solves to 1e-6."""
    # big enough that the fused levels run on many blocks (a single block never waits)
    cfg = configs.cantilever(96, 48, 48)
    ctx = rb.Context(0)
    G = _grid(ctx, cfg)
    try:
        for lvl in range(1, G.n_grid() - 1):
            rb._capi.check(rb.lib().rt_set_level_fused(G.handle, lvl, 1), ctx.handle)
        G[0].setForce(cfg["fload"].ravel())
        rb._capi.check(rb.lib().rt_ctx_set_wait_limit(ctx.handle, 0), ctx.handle)
        G[0].reset_displacement()
        with pytest.raises(rb.RTError) as ei:
            G.pcg(1e-6, 50)
        assert "grid barrier" in str(ei.value)
        rb._capi.check(rb.lib().rt_ctx_set_wait_limit(ctx.handle, -1), ctx.handle)
        G[0].reset_displacement()
        info = G.pcg(1e-6, 500)
        assert info.status == 0 and info.rel_residual <= 1e-6
    finally:
        G.close()
        ctx.close()


@pytest.mark.parametrize("where", ["force", "displacement", "density"])
def test_non_finite_input_reports_nan(where):
    cfg = configs.worst_case_box(24, 16, 12, seed=1)
    ctx = rb.Context(0)
    G = _grid(ctx, cfg)
    try:
        nv = G[0].nv
        f = np.zeros(3 * nv)
        f[2 * nv + cfg["load_nodes"]] = 1.0
        u = np.zeros(3 * nv)
        node = int(cfg["load_nodes"][len(cfg["load_nodes"]) // 2])
        if where == "force":
            f[node] = np.nan
        elif where == "displacement":
            u[node] = np.inf
        else:
            rho = cfg["rho"].ravel().copy()
            rho[rho.size // 2] = np.nan
            G[0].setRho(rho)
            G.update_stencil()
        G[0].setForce(f)
        G[0].setDisplacement(u)
        with pytest.raises(rb.RTError) as ei:
            G.pcg(1e-6, 100)
        assert ei.value.status == rb._capi.RT_ENAN, str(ei.value)
        # the context still works: a clean solve on a fresh hierarchy of the same context
        G.close()
        G = _grid(ctx, cfg)
        f[np.isnan(f)] = 0.0
        G[0].setForce(f)
        G[0].reset_displacement()
        assert G.pcg(1e-6, 500).status == 0
    finally:
        G.close()
        ctx.close()
