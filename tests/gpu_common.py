"""Shared set-up for the GPU parity tests: one CUDA hierarchy (through the C ABI)
and one CPU-oracle hierarchy built from the same seeded configuration."""
import numpy as np

import oracle as O
import robtop_b200 as rb
from robtop_b200 import configs

E, NU, P = 1e6, 0.4, 3.0


def build_pair(cfg, skip=True, precision=rb.FP64, smoother=rb.SMOOTH_SGS, pre=1, post=1, omega=0.6):
    ctx = rb.Context(0)
    params = rb.default_params(mode=cfg["mode"], skip_layer1=int(skip), youngs_modulus=E, poisson_ratio=NU,
                               power_penalty=P, min_rho=1e-3, precision=precision, smoother=smoother,
                               pre_sweeps=pre, post_sweeps=post, jacobi_omega=omega)
    G = rb.HierarchyGrid(ctx, params)
    G.genFromBox(cfg["eact"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    ws = cfg["mode"] in (rb.MODE_WSCF, rb.MODE_WSFF)
    if cfg["load_nodes"] is not None and len(cfg["load_nodes"]):
        G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"] if ws else None, p=P, E=E, nu=NU, skip=skip,
                    no_support=not ws)
    return ctx, G, H


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)


CONFIGS = {
    "cantilever": lambda: configs.cantilever(24, 12, 12),
    "worstcase": lambda: configs.worst_case_box(20, 16, 12, seed=3),
    "ragged_arch": lambda: configs.arch(27, 16, 14, tunnel=6, pad=3),
    # 48 nodes in x (a multiple of 16): the TMA-staged finest-level kernel runs on it
    "arch_x48": lambda: configs.arch(47, 18, 14, tunnel=7, pad=3),
    "free_nsff": lambda: configs.free_block(20, 12, 10, seed=4, mode=rb.MODE_NSFF),
    "free_nscf": lambda: configs.free_block(18, 12, 10, seed=5, mode=rb.MODE_NSCF),
}
