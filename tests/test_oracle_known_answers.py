"""Pins the CPU oracle with the reference's own known-answer tests.

The reference ships no golden vectors; these are the checks it defines:
  * test_rigid_displacement (optimization/optimization.cpp:697-709): K u_rigid = 0
  * selfTest BitSAT rank on a 0xAAAAAAAA pattern (optimization/optimization.cu:231-280)
  * verifyModifiedPM / aggregatedSystem (utils/test_utils.cpp:1249-1296, 1499-1568):
    the modified power method's eigenvalue equals the dense lambda_max of the
    aggregated compliance matrix C = [K^-1]_{L,L}
plus mathematical identities of the method (KE null space, R = P^T,
Galerkin coarse operators annihilate coarse rigid modes, coarsest
pseudo-inverse equals an SVD minimum-norm solve as Eigen::BDCSVD::solve).
"""
import numpy as np
import pytest

import oracle as O
from robtop_b200 import configs


def rigid_modes(shape_nodes):
    nz, ny, nx = shape_nodes
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x, y, z = x.ravel().astype(float), y.ravel().astype(float), z.ravel().astype(float)
    nv = x.size
    modes = []
    for t in range(3):
        m = np.zeros((3, nv))
        m[t] = 1
        modes.append(m.ravel())
    # rotations omega x p
    for w in np.eye(3):
        m = np.stack([w[1] * z - w[2] * y, w[2] * x - w[0] * z, w[0] * y - w[1] * x])
        modes.append(m.ravel())
    return modes


def test_template_matrix_symmetric_psd_nullspace6():
    KE = O.template_matrix(1e6, 0.4, 1.0)
    assert np.allclose(KE, KE.T, atol=1e-9 * np.abs(KE).max())
    ev = np.linalg.eigvalsh(KE)
    assert np.sum(np.abs(ev) < 1e-9 * ev.max()) == 6
    assert ev.min() > -1e-9 * ev.max()


def test_template_matrix_scaling():
    # KE is linear in E and scales with h (trilinear hex: KE(h) = h * KE(1))
    K1 = O.template_matrix(1.0, 0.3, 1.0)
    assert np.allclose(O.template_matrix(7.0, 0.3, 1.0), 7 * K1)
    assert np.allclose(O.template_matrix(1.0, 0.3, 2.0), 2 * K1)


def test_bitsat_rank_pattern():
    # 10000 words of 0xAAAAAAAA: every odd bit set; rank(i) = 16*(i//32) + (i%32)//2
    bits = np.full(10000, 0xAAAAAAAA, np.uint32)
    q = np.arange(0, 10000 * 32, 37, dtype=np.int64)
    r = O.bitsat_rank(bits, q)
    assert np.array_equal(r, 16 * (q // 32) + (q % 32) // 2)
    assert O.bits_total(bits) == 160000


@pytest.mark.parametrize("mode_ws", [False, True])
def test_rigid_displacement_nullspace(mode_ws):
    nx, ny, nz = 11, 8, 6
    eact = np.ones((nz, ny, nx), np.uint8)
    rho = configs.smoothed_density(eact.shape, 1, sigma=1.0)
    H = O.Hierarchy(eact, rho, None, p=3, E=1e6, nu=0.4)
    shape = (nz + 1, ny + 1, nx + 1)
    for m in rigid_modes(shape):
        r = np.zeros_like(m)
        H.arrs[0]["u"][:] = m
        H.arrs[0]["f"][:] = 0
        O.lib().or_fine_residual(H.lv(0), O.ptr(H.KE), O.ptr(H.arrs[0]["u"]), O.ptr(H.arrs[0]["f"]), O.ptr(r))
        scale = np.abs(H.applyK(np.random.default_rng(0).standard_normal(m.size))).max()
        assert np.abs(r).max() < 1e-9 * scale * np.abs(m).max()


def _small_hier(ws=True, nx=12, ny=8, nz=8, skip=False, seed=2):
    eact = np.ones((nz, ny, nx), np.uint8)
    rho = configs.smoothed_density(eact.shape, seed, sigma=1.5)
    vfix = None
    if ws:
        vfix = np.zeros((nz + 1, ny + 1, nx + 1), np.uint8)
        vfix[:, :, 0] = 1
    H = O.Hierarchy(eact, rho, vfix, p=3, E=1e6, nu=0.4, skip=skip)
    H.update_stencil()
    return H


def test_restriction_is_prolongation_transpose():
    H = _small_hier(ws=False, nx=16, ny=12, nz=12)
    rng = np.random.default_rng(0)
    for i in range(1, H.nlev):
        nvf = H.arrs[i - 1]["u"].size
        nvc = H.arrs[i]["u"].size
        uf = rng.standard_normal(nvf) * np.tile(H.arrs[i - 1]["vact"], 3)
        vc = rng.standard_normal(nvc) * np.tile(H.arrs[i]["vact"], 3)
        Ruf = np.zeros(nvc)
        O.lib().or_restrict(H.lv(i - 1), H.lv(i), O.ptr(uf), O.ptr(Ruf))
        Pvc = np.zeros(nvf)
        O.lib().or_prolong_add(H.lv(i - 1), H.lv(i), O.ptr(vc), O.ptr(Pvc))
        assert np.isclose(Ruf @ vc, uf @ Pvc, rtol=1e-12)


@pytest.mark.parametrize("skip", [False, True])
def test_galerkin_annihilates_coarse_rigid_modes(skip):
    # without supports: P maps coarse rigid modes to fine rigid modes, so A_c r_c = 0
    H = _small_hier(ws=False, nx=16, ny=16, nz=16, skip=skip)
    for i in range(1, H.nlev):
        L = H.levels[i]
        shape = (L.nz + 1, L.ny + 1, L.nx + 1)
        for m in rigid_modes(shape):
            out = np.zeros_like(m)
            O.lib().or_st_applyA(H.lv(i), O.ptr(np.ascontiguousarray(m)), O.ptr(out))
            st = H.arrs[i]["st"]
            assert np.abs(out).max() < 1e-8 * np.abs(st).max() * max(1.0, np.abs(m).max())


def test_galerkin_equals_ptap_dense():
    # the first coarse stencil equals P^T K P built densely from the fine operator
    H = _small_hier(ws=True, nx=8, ny=8, nz=8, skip=False)
    nvf = H.arrs[0]["u"].size
    nvc = H.arrs[1]["u"].size
    K = np.zeros((nvf, nvf))
    # Dirichlet form of the reference's restriction: fixed rows/cols dropped,
    # 1e6 * (number of incident elements) on the fixed diagonal
    L0 = H.levels[0]
    vfix = H.arrs[0]["vfix"]
    for j in range(nvf):
        e = np.zeros(nvf)
        e[j] = 1
        K[:, j] = H.applyK(e)
    nn = nvf // 3
    fixed = np.tile(vfix.astype(bool), 3)
    K[fixed, :] = 0
    K[:, fixed] = 0
    ne = np.zeros(nn)
    eact = H.arrs[0]["eact"]
    for z in range(L0.nz + 1):
        for y in range(L0.ny + 1):
            for x in range(L0.nx + 1):
                c = 0
                for i in range(8):
                    ex, ey, ez = x + i % 2 - 1, y + i // 2 % 2 - 1, z + i // 4 - 1
                    if 0 <= ex < L0.nx and 0 <= ey < L0.ny and 0 <= ez < L0.nz:
                        c += eact[ez, ey, ex]
                ne[x + (L0.nx + 1) * (y + (L0.ny + 1) * z)] = c
    for idx in np.flatnonzero(fixed):
        K[idx, idx] = 1e6 * ne[idx % nn]
    P = np.zeros((nvf, nvc))
    for j in range(nvc):
        e = np.zeros(nvc)
        e[j] = 1
        col = np.zeros(nvf)
        O.lib().or_prolong_add(H.lv(0), H.lv(1), O.ptr(e), O.ptr(col))
        P[:, j] = col
    Ac = P.T @ K @ P
    Ad = np.zeros((nvc, nvc))
    for j in range(nvc):
        e = np.zeros(nvc)
        e[j] = 1
        out = np.zeros(nvc)
        O.lib().or_st_applyA(H.lv(1), O.ptr(e), O.ptr(out))
        Ad[:, j] = out
    act = np.tile(H.arrs[1]["vact"].astype(bool), 3)
    assert np.allclose(Ad[np.ix_(act, act)], Ac[np.ix_(act, act)], rtol=1e-10, atol=1e-9 * np.abs(Ac).max())


@pytest.mark.parametrize("ws", [True, False])
def test_coarsest_pseudo_inverse_matches_svd(ws):
    # uniform density keeps the coarsest matrix well conditioned so the two
    # solves can be compared entry by entry
    nx = ny = nz = 8
    eact = np.ones((nz, ny, nx), np.uint8)
    vfix = None
    if ws:
        vfix = np.zeros((nz + 1, ny + 1, nx + 1), np.uint8)
        vfix[:, :, 0] = 1
    H = O.Hierarchy(eact, np.full(eact.shape, 0.5, np.float32), vfix, p=3, E=1e6, nu=0.4, skip=False)
    H.update_stencil()
    last = H.nlev - 1
    d = H.arrs[last]
    nv = d["u"].size // 3
    act = d["vact"].astype(bool)
    # dense coarsest matrix
    n = int(act.sum()) * 3
    A = np.zeros((3 * nv, 3 * nv))
    for j in range(3 * nv):
        e = np.zeros(3 * nv)
        e[j] = 1
        out = np.zeros(3 * nv)
        O.lib().or_st_applyA(H.lv(last), O.ptr(e), O.ptr(out))
        A[:, j] = out
    sel = np.tile(act, 3)
    As = A[np.ix_(sel, sel)]
    f = np.random.default_rng(1).standard_normal(3 * nv) * np.tile(act, 3)
    d["f"][:] = f
    O.lib().or_coarsest_solve(H.lv(last))
    u = d["u"][sel]
    # numpy SVD minimum-norm least squares, the meaning of Eigen::BDCSVD::solve
    u_ref = np.linalg.pinv(As, rcond=np.finfo(float).eps * n) @ f[sel]
    assert np.allclose(u, u_ref, rtol=1e-6, atol=1e-8 * np.abs(u_ref).max())


def _worstcase_small(nx=8, ny=8, nz=8):
    cfg = configs.worst_case_box(nx, ny, nz, seed=5)
    cfg["rho"] = configs.smoothed_density(cfg["eact"].shape, 5, sigma=1.5)
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    H.update_stencil()
    return cfg, H


def _aggregated_lambda(cfg, H):
    """aggregatedSystem (utils/test_utils.cpp:1499-1568): C = [K^-1]_{L,L} column by column."""
    nv = H.arrs[0]["u"].size // 3
    L = cfg["load_nodes"]
    cols = []
    for i in L:
        for c in range(3):
            b = np.zeros(3 * nv)
            b[c * nv + i] = 1
            x, it, rr = H.pcg(b, tol=1e-12, maxit=500)
            cols.append(np.concatenate([x[0 * nv + L], x[1 * nv + L], x[2 * nv + L]]))
    Cm = np.array(cols).T  # rows ordered (comp, node), cols ordered (node, comp)
    nl = L.size
    perm = np.array([c * nl + i for i in range(nl) for c in range(3)])
    Cm = Cm[perm, :]
    Cm = 0.5 * (Cm + Cm.T)
    return np.linalg.eigvalsh(Cm).max()


def test_modified_pm_matches_aggregated_compliance_eigenvalue():
    cfg, H = _worstcase_small()
    lam_dense = _aggregated_lambda(cfg, H)
    nl = cfg["load_nodes"].size
    fs = np.zeros(3 * nl)
    it = np.zeros(1, np.int32)
    lam = O.lib().or_modified_pm(H.LA, H.nlev, O.ptr(H.KE), nl, O.ptr(cfg["load_nodes"]),
                                 O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), 0, 0, None, None, 7, 500,
                                 O.ptr(it), O.ptr(fs))
    assert it[0] > 0
    assert abs(lam - lam_dense) / lam_dense < 2e-3  # PM stops at fch <= 1e-4 with one V-cycle per step


def test_lanczos_matches_aggregated_compliance_eigenvalue():
    cfg, H = _worstcase_small()
    lam_dense = _aggregated_lambda(cfg, H)
    nl = cfg["load_nodes"].size
    nv = H.arrs[0]["u"].size // 3
    k = 16
    work = np.zeros((k + 1) * 3 * nl + 10 * 3 * nv)
    lam = np.zeros(1)
    ritz = np.zeros(3 * nv)
    O.lib().or_lanczos(H.LA, H.nlev, O.ptr(H.KE), O.SMOOTH_SGS, 1, 1, 0.6, nl, O.ptr(cfg["load_nodes"]),
                       O.ptr(np.ascontiguousarray(cfg["normals"], np.float64)), 0, 0, None, 11, k, 1e-10, 500,
                       O.ptr(lam), O.ptr(ritz), O.ptr(work))
    assert abs(lam[0] - lam_dense) / lam_dense < 1e-5


def test_vcycle_and_pcg_converge():
    cfg = configs.cantilever(16, 8, 8)
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    H.update_stencil()
    b = cfg["fload"].ravel().copy()
    H.arrs[0]["f"][:] = b
    H.arrs[0]["u"][:] = 0
    rels = [H.vcycle(O.SMOOTH_GS, 1, 1) for _ in range(8)]
    assert rels[-1] < 1e-3 and all(rels[i + 1] < rels[i] for i in range(len(rels) - 1))
    x, it, rr = H.pcg(b, tol=1e-6, smoother=O.SMOOTH_SGS)
    assert rr <= 1e-6 and it < 30
    x2, it2, rr2 = H.pcg(b, tol=1e-6, smoother=O.SMOOTH_JACOBI, npre=2, npost=2, omega=0.6)
    assert rr2 <= 1e-6
    assert np.isclose(b @ x, b @ x2, rtol=1e-5)


def test_chebyshev_bound_estimate_matches_dense_spectrum():
    """The smoother bound lambda_max(D^-1 A) of the smoothed levels, estimated by 30 Lanczos steps
    in the A inner product, is a lower bound within 0.5 % of the dense spectrum's maximum on a
    high-contrast density (the 2-norm ratio |D^-1 A x| of a plain power method is not a bound
    there, and its convergence at the dense top of the spectrum is slow)."""
    cfg = configs.worst_case_box(10, 8, 6, seed=4)
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    H.update_stencil()
    for lvl in range(H.nlev - 1):
        d = H.arrs[lvl]
        n = d["u"].size
        free = np.ones(n, bool)
        if lvl == 0:
            free &= np.tile(~cfg["vfix"].ravel().astype(bool), 3)
        free &= np.tile(d["vact"].astype(bool), 3)
        cols = []
        zero = np.zeros(n)
        for j in np.flatnonzero(free):
            e = np.zeros(n)
            e[j] = 1.0
            r = np.zeros(n)
            z = np.zeros(n)
            if lvl == 0:
                O.lib().or_fine_residual(H.lv(0), O.ptr(H.KE), O.ptr(e), O.ptr(zero), O.ptr(r))
                O.lib().or_fine_jacobi(H.lv(0), O.ptr(H.KE), O.ptr(z), O.ptr(r), 1.0, O.ptr(d["r"]))
            else:
                O.lib().or_st_residual(H.lv(lvl), O.ptr(e), O.ptr(zero), O.ptr(r))
                O.lib().or_st_jacobi(H.lv(lvl), O.ptr(z), O.ptr(r), 1.0, O.ptr(d["r"]))
            cols.append(-z[free])
        M = np.array(cols).T  # D^-1 A on the free degrees of freedom
        lam = np.max(np.linalg.eigvals(M).real)
        est = H.LA[lvl].lmax
        assert est <= lam * (1 + 1e-9), (lvl, est, lam)
        assert est >= 0.995 * lam, (lvl, est, lam)


def test_surface_rule_numpy_and_c_agree():
    rng = np.random.default_rng(3)
    eact = (rng.random((7, 6, 9)) < 0.6).astype(np.uint8)
    s_c = O.surface_nodes(eact)
    s_np = configs.surface_nodes(eact).astype(np.uint8)
    assert np.array_equal(s_c, s_np)
    assert np.array_equal(O.node_active(eact).astype(bool), configs.node_active(eact))


def test_cube_occupancy_matches_dense_chain():
    # the reference's cubic bit hierarchy and the dense-box chain describe the same solids
    R = 16
    rng = np.random.default_rng(4)
    dense = (rng.random((R, R, R)) < 0.3).astype(np.uint8)
    bits = np.packbits(dense.ravel(), bitorder="little").view(np.uint32)
    levels = O.cube_hierarchy(R, bits)
    cur = dense
    for Rl, eb, vb in levels:
        d = np.unpackbits(eb.view(np.uint8), bitorder="little")[: Rl ** 3].reshape(Rl, Rl, Rl)
        assert np.array_equal(d, cur)
        v = np.unpackbits(vb.view(np.uint8), bitorder="little")[: (Rl + 1) ** 3].reshape(Rl + 1, Rl + 1, Rl + 1)
        assert np.array_equal(v.astype(bool), configs.node_active(cur))
        cur = O.coarsen_elements(cur, 2)
    assert O.bits_total(levels[-1][1]) <= 400 < O.bits_total(levels[-2][1])


def test_gs_maps_padding_and_order():
    R = 5
    rng = np.random.default_rng(6)
    dense = (rng.random((R, R, R)) < 0.5).astype(np.uint8)
    bits = np.packbits(dense.ravel(), bitorder="little").view(np.uint32)
    vb = O.cube_vbits(R, bits)
    vl, gs_num, ngs = O.gs_maps(R + 1, vb)
    assert all(g % 32 == 0 for g in gs_num) and ngs == gs_num.sum()
    assert len(set(vl.tolist())) == vl.size


def test_voxeliser_resolution_rule_and_volumes():
    """The oracle voxeliser (voxelizer/cpu_voxelizer.cpp:245-322 restated): the cube resolution
    is the first power of two above prefer_reso (voxelize_main.cpp:312-340), and the solid
    voxel volume of closed meshes matches their enclosed volume."""
    from robtop_b200 import configs

    for prefer, R in ((1, 2), (7, 8), (31, 32), (63, 64), (64, 128), (200, 256)):
        assert O.voxel_box(np.zeros((1, 3), np.float32) + [[0, 0, 0]], prefer)[0] == R
    cases = {"sphere": (configs.icosphere(4), None), "torus": (configs.torus(1.0, 0.35, 64, 32), None),
             "box": (configs.box_mesh((0, 0, 0), (1.0, 0.5, 0.7)), 0.35)}
    for name, ((v, f), exact) in cases.items():
        d = v.astype(np.float64)[f]
        poly = abs(np.einsum("ij,ij->i", d[:, 0], np.cross(d[:, 1], d[:, 2])).sum()) / 6.0  # enclosed volume
        if exact is not None:
            assert abs(poly - exact) < 1e-6
        R, bmin, bmax, unit = O.voxel_box(v, 127)
        bits = O.voxelize_solid(v, f, R, bmin, unit)
        vol = O.bits_total(bits) * float(unit[0]) ** 3
        assert abs(vol - poly) < 0.02 * poly, (name, vol, poly)


def test_voxeliser_word_reverse_and_bit_order():
    """Bit id x + y R + z R^2 at bit 31 - id % 32 (most significant first); the word reverse
    (wordReverse_g) gives the hierarchy's least-significant-first layout."""
    from robtop_b200 import configs

    v, f = configs.icosphere(2, (0.0, 0.0, 0.0), 1.0)
    R, bmin, bmax, unit = O.voxel_box(v, 31)
    msb = O.voxelize_solid(v, f, R, bmin, unit)
    lsb = O.word_reverse(msb)
    np.testing.assert_array_equal(O.word_reverse(lsb), msb)
    # least-significant-first: bit id % 32 of word id / 32; the centred sphere fills the cube's
    # centre, not its corner, and is mirror-symmetric in x up to a thin shell of boundary voxels
    ids = np.arange(R ** 3)
    vol = ((lsb[ids >> 5] >> (ids & 31)) & 1).reshape(R, R, R)  # [z][y][x]
    assert vol[R // 2, R // 2, R // 2] == 1 and vol[0, 0, 0] == 0
    assert np.count_nonzero(vol != vol[:, :, ::-1]) < 0.05 * vol.sum()


def test_mma_reaches_the_separable_optimum():
    """The oracle's MMA (or_mma.c, optimization/mma_t.cu's method with one constraint) on
    min sum c_j / x_j / n s.t. 1e3 (mean(x) - V) <= 0, 0.01 <= x <= 1: 80 steps reach the known
    optimum x_j = V n sqrt(c_j) / sum sqrt(c) (inside the bounds here) to 1e-12, and each step's
    design satisfies the subproblem's stationarity: between its move bounds, the derivative of
    the approximated Lagrangian vanishes."""
    rng = np.random.default_rng(0)
    n, V = 1000, 0.3
    c = rng.uniform(0.5, 2.0, n)
    m = O.MMA(n, 0.01, 1.0)
    for it in range(80):
        x0, low, upp, a, b = m.x.copy(), m.low.copy(), m.upp.copy(), m.alpha.copy(), m.beta.copy()
        df, dg = -c / x0 ** 2 / n, np.full(n, 1e3 / n)
        lam = m.update(df, dg, 1e3 * (x0.mean() - V))
        if it < 5:
            # p, q of both functions at x0 (mma_t.cu:70-81), then d/dx of sum (p0 + lam p1) / (U - x)
            # + (q0 + lam q1) / (x - L) at the new design, zero where it is strictly inside [a, b]
            r = 1e-5 / 0.99
            pq = lambda f: ((upp - x0) ** 2 * (1.001 * np.maximum(f, 0) + 0.001 * np.maximum(-f, 0) + r),
                            (x0 - low) ** 2 * (0.001 * np.maximum(f, 0) + 1.001 * np.maximum(-f, 0) + r))
            (p0, q0), (p1, q1) = pq(df), pq(dg)
            xn = m.x
            grad = (p0 + lam * p1) / (upp - xn) ** 2 - (q0 + lam * q1) / (xn - low) ** 2
            inside = (xn > a + 1e-12) & (xn < b - 1e-12)
            scale = np.abs((p0 + lam * p1) / (upp - xn) ** 2).max()
            assert np.abs(grad[inside]).max() <= 1e-9 * scale, it
    xs = V * n * np.sqrt(c) / np.sqrt(c).sum()
    assert np.abs(m.x - xs).max() <= 1e-12


def test_mma_step_solves_the_subproblem_the_reference_poses():
    """One step of the oracle's MMA equals the optimum of the subproblem as the reference states
    it (optimization/mma_t.cu:70-89, mma_t.h:229-237: a0 = 1, a = 0, c = 10, d = 1), solved here
    by a general constrained optimiser over (x, y, z) instead of the one-multiplier dual: the
    dual's design is feasible, its objective is not above the optimiser's (to 1e-9 relative),
    and the designs agree to 1e-4, for an active and an inactive constraint."""
    from scipy.optimize import minimize

    rng = np.random.default_rng(4)
    n = 40
    for target in (0.3, 0.9):  # volume constraint active / inactive at the start design
        m = O.MMA(n, 0.01, 1.0)
        x0, low, upp, a, b = m.x.copy(), m.low.copy(), m.upp.copy(), m.alpha.copy(), m.beta.copy()
        c = rng.uniform(0.5, 2.0, n)
        df, dg = -c / x0 ** 2 / n, np.full(n, 1e3 / n)
        g = 1e3 * (x0.mean() - target)
        lam = m.update(df, dg, g)
        r = 1e-5 / 0.99
        pq = lambda f: ((upp - x0) ** 2 * (1.001 * np.maximum(f, 0) + 0.001 * np.maximum(-f, 0) + r),
                        (x0 - low) ** 2 * (0.001 * np.maximum(f, 0) + 1.001 * np.maximum(-f, 0) + r))
        (p0, q0), (p1, q1) = pq(df), pq(dg)
        bb = np.sum(p1 / (upp - x0) + q1 / (x0 - low)) - g
        f0 = lambda v: np.sum(p0 / (upp - v[:n]) + q0 / (v[:n] - low)) + v[n + 1] + 10 * v[n] + 0.5 * v[n] ** 2
        con = {"type": "ineq", "fun": lambda v: bb - (np.sum(p1 / (upp - v[:n]) + q1 / (v[:n] - low)) - v[n])}
        bounds = list(zip(a, b)) + [(0, None), (0, None)]
        res = minimize(f0, np.concatenate([x0, [0.0, 0.0]]), method="SLSQP", bounds=bounds, constraints=[con],
                       options={"ftol": 1e-12, "maxiter": 2000})
        y = max(0.0, lam - 10.0)
        mine = np.concatenate([m.x, [y, 0.0]])
        assert con["fun"](mine) >= -1e-9 * abs(bb)
        assert f0(mine) <= res.fun + 1e-9 * abs(res.fun), (target, f0(mine), res.fun)
        assert np.abs(res.x[:n] - m.x).max() <= 1e-4, (target, np.abs(res.x[:n] - m.x).max())
