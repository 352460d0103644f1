"""The projection API (optimization/projection.h:16-65), Grid::elementCompliance
(grid/Grid.cu:3434-3480) and the design-state files with checkpoint / resume of the
optimisation loop, on the GPU, against the oracle where it has the same function."""
import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from robtop_b200 import configs
from robtop_b200 import optimization as opt

from gpu_common import CONFIGS, build_pair, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cantilever", "ragged_arch", "free_nsff", "free_nscf"])
def test_force_and_displacement_projection(name):
    cfg = CONFIGS[name]()
    ctx, G, H = build_pair(cfg)
    try:
        nv = G[0].nv
        f = np.random.default_rng(3).standard_normal(3 * nv) * np.tile(G[0].getVact(), 3)
        pf = G.forceProject(f)
        ln = cfg["load_nodes"]
        nl = ln.size
        constrain = 1 if cfg["mode"] in (rb.MODE_WSCF, rb.MODE_NSCF) else 0
        ws = cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF)
        pos = np.stack(np.unravel_index(ln, cfg["vfix"].shape)[::-1], 1).astype(np.float64)
        Rd = np.zeros(6 * 3 * nl)
        normals = np.ascontiguousarray(cfg["normals"], np.float64)
        nrig = 0 if ws else O.lib().or_rigid_basis(nl, O.ptr(np.ascontiguousarray(pos)), O.ptr(normals), constrain,
                                                    O.ptr(Rd))
        fo = f.copy()
        O.lib().or_force_project(nv, nl, O.ptr(np.ascontiguousarray(ln, np.int32)), O.ptr(normals), constrain, nrig,
                                 O.ptr(Rd) if nrig else None, O.ptr(fo))
        assert rel_err(pf, fo) < 1e-12
        # P is a projection, and only load nodes carry force
        assert rel_err(G.forceProject(pf), pf) < 1e-12
        mask = np.zeros(nv, bool)
        mask[ln] = True
        assert np.all(pf.reshape(3, nv)[:, ~mask] == 0)
        # support force round trip
        assert np.array_equal(G.getLoadNodes(), np.sort(ln))
        fs = G.getForceSupport(pf)
        assert fs.shape == (3, nl)
        assert np.array_equal(G.setForceSupport(fs), pf)
        # displacement projection: orthogonal to the rigid modes without supports, identity with them
        u = np.random.default_rng(4).standard_normal(3 * nv) * np.tile(G[0].getVact(), 3)
        pu = G.displacementProject(u)
        if ws:
            assert np.array_equal(pu, u)
        else:
            Ru = np.zeros(6 * 3 * nv)
            O.lib().or_rigid_nodes(H.lv(0), O.ptr(Ru))
            uo = u.copy()
            O.lib().or_displacement_project(nv, O.ptr(Ru), O.ptr(uo))
            assert rel_err(pu, uo) < 1e-10
            assert np.abs(Ru.reshape(6, -1) @ pu).max() < 1e-9 * np.linalg.norm(u)
    finally:
        G.close()
        ctx.close()


def test_element_compliance_sums_to_uKu():
    cfg = CONFIGS["worstcase"]()
    ctx, G, H = build_pair(cfg)
    try:
        G.update_stencil()
        nv = G[0].nv
        u = np.random.default_rng(5).standard_normal(3 * nv) * np.tile(G[0].getVact(), 3) * 1e-3
        ce = G[0].elementCompliance(u)
        G[0].setDisplacement(u)
        Ku = G[0].applyK(u)
        # fixed nodes enter K u as identity rows: compare on a displacement zero at the supports
        free = np.tile(1 - cfg["vfix"].ravel().astype(np.float64), 3)
        u0 = u * free
        ce0 = G[0].elementCompliance(u0)
        assert abs(ce0.sum() - u0 @ G[0].applyK(u0)) <= 1e-5 * abs(u0 @ G[0].applyK(u0))
        # per element: -rho / p times the sensitivity of the same displacement
        rb._capi.check(rb.lib().rt_sensitivity(G.handle, 0), ctx.handle)
        s = G[0].getSens()
        rho = cfg["rho"].ravel()
        assert rel_err(ce, -rho / 3.0 * s) < 1e-5
        assert np.all(ce >= -1e-12)
        del Ku
    finally:
        G.close()
        ctx.close()


def test_state_files_and_resumed_optimisation(tmp_path):
    """Checkpoints every 2 OC iterations; resuming from the iteration-2 checkpoint reproduces the
    uninterrupted run's eigenvalues and densities (deterministic kernels, fixed Lanczos seed)."""
    cfg = configs.cantilever(24, 12, 12)

    def setup():
        opt.setParameters(0.4, 0.0, 0.03, 2, 0.5, 3.0, 1e-3, 32, 1e6, 0.4)
        opt.setWorkMode("wsff")
        nx, ny, nz = 24, 12, 12
        opt.setBoundaryCondition(lambda p: p[0] == 0.0, lambda p: p[0] == nx and p[2] == 0.0,
                                 lambda p: (0.0, 0.0, -1.0))
        R = 32
        bits = np.zeros((R ** 3 + 31) // 32, np.uint32)
        for z in range(nz):
            for y in range(ny):
                t = np.arange(nx) + R * (y + R * z)
                np.bitwise_or.at(bits, t >> 5, (np.uint32(1) << (t & 31).astype(np.uint32)))
        opt.buildGrids(bits, R)
        opt.uploadTemplateMatrix()

    worst = lambda: opt.worstCaseLanczos(8, 1e-8, seed=3)  # noqa: E731
    setup()
    opt.setOutpurDir(str(tmp_path))
    full = opt.optimization(max_iter=4, worst=worst, checkpoint_every=2)
    rho_full = opt.getGrids()[0].getRho()
    assert len(full) == 4
    man = opt.getGrids().read_state(str(tmp_path / "iter_2"))
    assert man["meta"]["iteration"] == 2 and len(man["meta"]["records"]) == 2
    setup()
    resumed = opt.optimization(max_iter=4, worst=worst, resume=str(tmp_path / "iter_2"))
    assert np.allclose(resumed, full, rtol=1e-12, atol=0)
    assert np.array_equal(opt.getGrids()[0].getRho(), rho_full)
    # a state of another grid is refused
    G2 = rb.HierarchyGrid(rb.Context(0), rb.default_params(mode=cfg["mode"]))
    G2.genFromBox(configs.cantilever(20, 12, 12)["eact"])
    with pytest.raises(ValueError):
        G2.read_state(str(tmp_path / "iter_2"))
    G2.close()
