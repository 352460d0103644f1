"""The oracle pinned to the reference's own code (CPU part).

* KE: the oracle's or_template_matrix against the reference's initTemplateMatrix
  (element/templateMatrix.cpp:31-124), compiled from the reference sources into
  oracle/_ref/libref_ke.so where the reference is present, and against the fixture
  tests/golden/ref_template_matrix.npz that build wrote (tests/golden/make_ref_fixtures.py).
* The oracle's applyK, sensitivity, OC trial and filter against the outputs of the reference's
  own CUDA kernels (grid/Grid.cu:2439-2517, 2323-2409; optimization/optimization.cu:44-162) on
  seeded inputs, stored in tests/golden/ref_kernels.npz by the same script on a GPU machine.
* The optimisation loop's stop test against the reference's converge_criteria (utils/snippet.h)
  in both of its builds, and the oracle's solid voxeliser against the reference's CPU voxeliser
  (voxelizer/cpu_voxelizer.cpp), each as fixtures and against the live build.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O
from oracle import reference

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from ref_inputs import CASES, FILTER_RADIUS, OC, P, inputs  # noqa: E402

KE_FIXTURE = os.path.join(HERE, "golden", "ref_template_matrix.npz")
KERNEL_FIXTURE = os.path.join(HERE, "golden", "ref_kernels.npz")


def test_template_matrix_matches_reference_fixture():
    g = np.load(KE_FIXTURE)
    for (h, E, nu), ke in zip(g["params"], g["ke"]):
        assert np.array_equal(O.template_matrix(E, nu, h), ke), (h, E, nu)


@pytest.mark.skipif(not os.path.exists(reference.KE_LIB), reason="oracle/_ref/libref_ke.so not built")
def test_template_matrix_matches_reference_build():
    for h, E, nu in [(1.0, 1e6, 0.4), (2.0, 3.0, 0.1), (0.25, 7e4, 0.45)]:
        assert np.array_equal(O.template_matrix(E, nu, h), reference.template_matrix(h, E, nu)), (h, E, nu)


def _oracle_outputs(name):
    cfg, KE, u, sens, eshell, ws = inputs(name)
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"] if ws else None, p=P, E=1e6, nu=0.4, no_support=not ws)
    nz, ny, nx = cfg["eact"].shape
    eact = np.ascontiguousarray(cfg["eact"].ravel(), np.uint8)
    rho = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
    s = np.zeros(rho.size, np.float32)
    O.lib().or_sensitivity(nx, ny, nz, O.ptr(eact), O.ptr(rho), P, O.ptr(KE), O.ptr(u), O.ptr(s))
    oc = np.zeros_like(rho)
    O.lib().or_oc_try(rho.size, O.ptr(eact), O.ptr(eshell), O.ptr(rho), O.ptr(sens), OC["thres"], OC["step"],
                      OC["damp"], OC["rhomin"], O.ptr(oc))
    flt = np.zeros_like(rho)
    O.lib().or_filter(nx, ny, nz, O.ptr(eact), FILTER_RADIUS, O.ptr(sens), O.ptr(flt))
    return {"applyK": H.applyK(u), "sensitivity": s, "oc_try": oc, "filter": flt}, eact


@pytest.mark.skipif(not os.path.exists(KERNEL_FIXTURE), reason="tests/golden/ref_kernels.npz not generated")
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_kernel_outputs(name):
    g = np.load(KERNEL_FIXTURE)
    mine, eact = _oracle_outputs(name)
    ref = {k: g[f"{name}/{k}"] for k in ("applyK", "sensitivity", "oc_try", "filter")}
    # K u: the same FP64 sums in another order; the element weights rho^p come from C's powf here
    # and CUDA's in the reference, which may differ by an ulp (2^-24) where rho varies
    assert np.abs(mine["applyK"] - ref["applyK"]).max() <= 1e-6 * np.abs(ref["applyK"]).max()
    # sensitivities: the reference adds FP32 partial sums with atomicAdd (order varies), the oracle
    # sums in FP64 and rounds once
    act = eact.astype(bool)
    assert np.abs(mine["sensitivity"] - ref["sensitivity"]).max() <= 2e-6 * np.abs(ref["sensitivity"]).max()
    # the OC trial: FP32 powf in both, one rounding apart at most
    assert np.abs(mine["oc_try"][act] - ref["oc_try"][act]).max() <= 2e-6
    # the filter: FP32 weights, FP64 sums in both
    assert np.abs(mine["filter"][act] - ref["filter"][act]).max() <= 1e-6 * np.abs(ref["filter"]).max()


STOP_FIXTURE = os.path.join(HERE, "golden", "ref_stop.npz")


def _stop_flags(c, g, integer_abs):
    from robtop_b200.optimization import ConvergeCriteria

    crit = ConvergeCriteria(1, 2, 5e-3, integer_abs=integer_abs)
    return [int(crit.update(ci, [gi])) for ci, gi in zip(c, g)]


def test_stop_test_matches_reference_fixture():
    """optimization()'s stop test (ConvergeCriteria) gives the reference converge_criteria's
    update() results on the fixture's sequences, stop for stop, in both builds of the header
    (g++'s integer abs of the change, and the floating-point one)."""
    d = np.load(STOP_FIXTURE)
    for i in range(int(d["n"])):
        assert _stop_flags(d[f"c{i}"], d[f"g{i}"], True) == d[f"stop{i}"].tolist(), i
        assert _stop_flags(d[f"c{i}"], d[f"g{i}"], False) == d[f"stop_fabs{i}"].tolist(), i


@pytest.mark.skipif(not (os.path.exists(reference.STOP_LIB) and os.path.exists(reference.STOP_FABS_LIB)),
                    reason="oracle/_ref/libref_stop*.so not built")
def test_stop_test_matches_reference_build():
    rng = np.random.default_rng(5)
    for case in range(60):
        n = int(rng.integers(1, 30))
        scale = 10.0 ** rng.uniform(-4, 2)  # compliances both below and above 1
        c = scale * (3.0 + rng.uniform(0.01, 2.0) * rng.uniform(0.2, 0.97) ** np.arange(n))
        c *= 1 + rng.normal(0, 10 ** rng.uniform(-5, -2), n)
        g = [np.zeros(n), -0.4 * 0.05 * np.ones(n), 0.3 * (0.95 ** np.arange(1, n + 1) - 1)][case % 3]
        assert _stop_flags(c, g, True) == reference.converge_run(1, 2, 5e-3, c, g).tolist(), case
        assert _stop_flags(c, g, False) == reference.converge_run(1, 2, 5e-3, c, g, float_abs=True).tolist(), case


VOX_FIXTURE = os.path.join(HERE, "golden", "ref_vox.npz")


def test_voxeliser_matches_reference_fixture():
    """The oracle's solid voxeliser gives the reference CPU voxeliser's bits
    (voxelizer/cpu_voxelizer.cpp:262-322), bit for bit, on closed meshes (spheres, rotated
    sphere and torus, boxes on voxel centres and flat, merged spheres) at resolutions 8, 32, 64."""
    from make_ref_fixtures import VOX_PREFER, vox_meshes

    g = np.load(VOX_FIXTURE)
    for name, (v, f) in vox_meshes().items():
        for prefer in VOX_PREFER:
            R, bmin, bmax, unit = O.voxel_box(v, prefer)
            assert np.array_equal(O.voxelize_solid(v, f, R, bmin, unit), g[f"{name}/{prefer}"]), (name, prefer)


@pytest.mark.skipif(not os.path.exists(reference.VOX_LIB), reason="oracle/_ref/libref_vox.so not built")
def test_voxeliser_matches_reference_build():
    """The same against the live build, at 256^3 as well and on merged meshes of other sizes."""
    from make_ref_fixtures import vox_meshes

    from robtop_b200 import configs

    meshes = dict(vox_meshes())
    meshes["three_tori"] = configs.merge_meshes(configs.torus(1.0, 0.3, 48, 24),
                                                (configs.rigid_transform(configs.torus(0.6, 0.2, 32, 16)[0], 5),
                                                 configs.torus(0.6, 0.2, 32, 16)[1]))
    for name, (v, f) in meshes.items():
        for prefer in (15, 200):
            R, bmin, bmax, unit = O.voxel_box(v, prefer)
            assert np.array_equal(O.voxelize_solid(v, f, R, bmin, unit),
                                  reference.voxelize_solid(v, f, R, bmin, bmax)), (name, prefer)
