"""Seeded inputs of the reference-kernel fixtures (shared by the fixture script and the tests)."""
import numpy as np

import oracle as O
from robtop_b200 import configs

E, NU, P = 1e6, 0.4, 3.0
CASES = {
    "cantilever_24x12x12": lambda: configs.cantilever(24, 12, 12),
    "arch_27x16x14": lambda: configs.arch(27, 16, 14, tunnel=6, pad=3),
    "free_20x12x10": lambda: configs.free_block(20, 12, 10, seed=4),
}
OC = dict(thres=0.37, step=0.05, damp=0.5, rhomin=1e-3)
FILTER_RADIUS = 2.0


def inputs(name):
    """(cfg, KE, u, sens, eshell) for one case; u on the active nodes, sens <= 0 mostly."""
    cfg = CASES[name]()
    nz, ny, nx = cfg["eact"].shape
    nv = (nx + 1) * (ny + 1) * (nz + 1)
    vact = O.node_active(cfg["eact"]).ravel().astype(np.float64)
    rng = np.random.default_rng(1234)
    u = rng.standard_normal(3 * nv) * np.tile(vact, 3) * 1e-3
    sens = (-np.abs(rng.standard_normal(nx * ny * nz)) + 0.05).astype(np.float32) * cfg["eact"].ravel()
    eshell = (rng.random(nx * ny * nz) < 0.05).astype(np.uint8) * cfg["eact"].ravel()
    KE = O.template_matrix(E, NU, 1.0)
    ws = cfg["mode"] in (configs.MODE_WSCF, configs.MODE_WSFF)
    return cfg, KE, u, sens, eshell, ws
