"""The reference's own CUDA kernels, compiled from its sources for sm_100a
(oracle/_ref/libref_kernels.so, `make -C oracle ref`), against the oracle and against this
library on the same seeded inputs: applyK_OTFA_kernel (grid/Grid.cu:2439-2517),
computeSensitivity_kernel and trySensMultiplier_kernel (optimization/optimization.cu:44-162),
filterSensitivity_kernel (grid/Grid.cu:2323-2409)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from oracle import reference

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from ref_inputs import CASES, FILTER_RADIUS, OC, P, inputs  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(reference.KERNELS_LIB),
                                 reason="oracle/_ref/libref_kernels.so not built (needs the reference sources)")]


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_kernels_against_oracle_and_library(name):
    K = reference.Kernels()
    cfg, KE, u, sens, eshell, ws = inputs(name)
    vfix = cfg["vfix"] if ws else None
    nz, ny, nx = cfg["eact"].shape
    eact = np.ascontiguousarray(cfg["eact"].ravel(), np.uint8)
    act = eact.astype(bool)
    rho = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
    ref_f = K.apply_k(cfg["eact"], vfix, rho, P, KE, u)
    # this library's K u (FP64) through the C ABI: both evaluate the weights with CUDA's powf
    ctx = rb.Context(0)
    G = rb.HierarchyGrid(ctx, rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4,
                                                power_penalty=P, min_rho=1e-3))
    try:
        G.genFromBox(cfg["eact"])
        G[0].setRho(rho)
        if ws:
            G.set_support(cfg["vfix"])
        G.update_stencil()
        assert np.abs(G[0].applyK(u) - ref_f).max() <= 1e-12 * np.abs(ref_f).max()
        # the oracle with the same weights (C's powf may differ from CUDA's by an ulp)
        H = O.Hierarchy(cfg["eact"], cfg["rho"], vfix, p=P, E=1e6, nu=0.4, no_support=not ws)
        H.set_weights(G[0].getPenalty())
        assert np.abs(H.applyK(u) - ref_f).max() <= 1e-12 * np.abs(ref_f).max()
        ref_s = K.sensitivity(cfg["eact"], rho, P, KE, u)
        G[0].setDisplacement(u)
        rb._capi.check(rb.lib().rt_sensitivity(G.handle, 0), ctx.handle)
        assert np.abs(G[0].getSens() - ref_s).max() <= 2e-6 * np.abs(ref_s).max()
        ref_flt = K.filter(cfg["eact"], FILTER_RADIUS, sens)
        G[0].setSens(sens)
        G[0].filterSensitivity(FILTER_RADIUS)
        assert np.abs(G[0].getSens()[act] - ref_flt[act]).max() <= 1e-6 * np.abs(ref_flt).max()
        ref_oc = K.oc_try(cfg["eact"], eshell, rho, sens, OC["thres"], OC["step"], OC["damp"], OC["rhomin"])
        oc = np.zeros_like(rho)
        O.lib().or_oc_try(rho.size, O.ptr(eact), O.ptr(eshell), O.ptr(rho), O.ptr(np.ascontiguousarray(sens)),
                          OC["thres"], OC["step"], OC["damp"], OC["rhomin"], O.ptr(oc))
        assert np.abs(oc[act] - ref_oc[act]).max() <= 2e-6
    finally:
        G.close()
        ctx.close()
