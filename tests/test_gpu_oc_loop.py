"""Several OC iterations of the fixed-load optimisation (solveFEM, computeSensitivity,
filterSensitivity, updateDensities: optimization/optimization.cpp:583-673) on the GPU
against the same loop in the oracle: the density field stays within 1e-4 max-abs."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from gpu_common import CONFIGS, E, NU, P, build_pair

pytestmark = pytest.mark.gpu


def test_density_after_oc_iterations():
    cfg = CONFIGS["cantilever"]()
    ctx, G, H = build_pair(cfg)
    nz, ny, nx = cfg["eact"].shape
    eact = np.ascontiguousarray(cfg["eact"].ravel(), np.uint8)
    nact = int(eact.sum())
    b = np.ascontiguousarray(cfg["fload"].ravel(), np.float64)
    rho_g = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
    rho_o = rho_g.copy()
    lam, trials = C.c_float(), C.c_int()
    try:
        for it in range(3):
            # device: solve, sensitivity, filter (radius 2), OC update to volume 0.4
            G[0].setRho(rho_g)
            G.update_stencil()
            G[0].setForce(b)
            G[0].reset_displacement()
            info = G.pcg(1e-10, 1000)
            assert info.status == 0
            rb._capi.check(rb.lib().rt_sensitivity(G.handle, 0), ctx.handle)
            G[0].filterSensitivity(2.0)
            rb._capi.check(rb.lib().rt_oc_update(G.handle, 0.4, C.byref(lam), C.byref(trials)), ctx.handle)
            rho_g = np.ascontiguousarray(G[0].getRho(), np.float32)
            # oracle: the same steps in FP64 C
            Ho = O.Hierarchy(cfg["eact"], rho_o.reshape(cfg["eact"].shape), cfg["vfix"], p=P, E=E, nu=NU)
            Ho.update_stencil()
            x, _, _ = Ho.pcg(b, tol=1e-10, maxit=1000)
            s = np.zeros(rho_o.size, np.float32)
            O.lib().or_sensitivity(nx, ny, nz, O.ptr(eact), O.ptr(rho_o), P, O.ptr(Ho.KE), O.ptr(x), O.ptr(s))
            fs = np.zeros_like(s)
            O.lib().or_filter(nx, ny, nz, O.ptr(eact), 2.0, O.ptr(s), O.ptr(fs))
            tmp = np.zeros_like(rho_o)
            its = np.zeros(1, np.int32)
            O.lib().or_oc_update(rho_o.size, O.ptr(eact), None, O.ptr(rho_o), O.ptr(fs), 0.4, 0.03, 0.5, 1e-3, nact,
                                 O.ptr(its), O.ptr(tmp))
            assert np.abs(rho_g - rho_o).max() <= 1e-4, f"iteration {it}"
        assert np.abs(rho_g - cfg["rho"].ravel()).max() > 1e-2  # the design moved
    finally:
        G.close()
        ctx.close()
