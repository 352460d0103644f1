"""Writes tests/golden/c2_lanczos.npz: the oracle's worst-case eigenvalue of the 128x128x64
worst-case box (smoothed random density, seed 0; z = 0 clamped; top face loadable, wsff),
Lanczos with k = 16 Krylov vectors from the seeded start vector 100, inner plain FP64
SGS V-cycle PCG solves to relative residual 1e-9, and the Ritz load on the load nodes.

The oracle is the CPU restatement of the reference algorithm (oracle/rt_oracle.c); this
fixture lets the GPU tests compare the full-size configuration without running the oracle
for minutes in every test session.  Run from the repository root:
    python tests/golden/make_c2_lanczos.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from robtop_b200 import configs  # noqa: E402

NX, NY, NZ, SEED, START, K, TOL = 128, 128, 64, 0, 100, 16, 1e-9


def main():
    cfg = configs.worst_case_box(NX, NY, NZ, seed=SEED)
    t0 = time.perf_counter()
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    H.update_stencil()
    nv = H.arrs[0]["u"].size // 3
    nl = cfg["load_nodes"].size
    work = np.zeros((K + 1) * 3 * nl + 10 * 3 * nv)
    lam = np.zeros(1)
    ritz = np.zeros(3 * nv)
    inner = O.lib().or_lanczos(H.LA, H.nlev, O.ptr(H.KE), O.SMOOTH_SGS, 1, 1, 0.6, nl, O.ptr(cfg["load_nodes"]),
                               O.ptr(np.ascontiguousarray(cfg["normals"])), 0, 0, None, START, K, TOL, 2000,
                               O.ptr(lam), O.ptr(ritz), O.ptr(work))
    ln = cfg["load_nodes"]
    load = np.stack([ritz[c * nv + ln] for c in range(3)])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_lanczos.npz")
    np.savez_compressed(out, lam=lam[0], load=load, load_nodes=ln, dims=np.array([NX, NY, NZ]), seed=SEED,
                        start=START, k=K, inner_tol=TOL, inner_iterations=inner)
    print(f"lambda {lam[0]:.15e}, {inner} inner PCG iterations, {time.perf_counter() - t0:.0f} s -> {out}")


if __name__ == "__main__":
    main()
