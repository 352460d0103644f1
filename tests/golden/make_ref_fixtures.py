"""Writes the fixtures that pin the oracle to the reference's own code:

* ref_template_matrix.npz: KE from the reference's initTemplateMatrix
  (element/templateMatrix.cpp:31-124, built into oracle/_ref/libref_ke.so by `make -C oracle ref`)
  for three (h, E, nu);
* ref_stop.npz: the update() results of the reference's converge_criteria (utils/snippet.h:156-213,
  oracle/_ref/libref_stop.so and libref_stop_fabs.so: integer and floating-point abs of the change)
  on the seeded sequences of stop_sequences() below;
* ref_vox.npz: the solid bits of the reference's CPU voxeliser (voxelizer/cpu_voxelizer.cpp:262-322,
  oracle/_ref/libref_vox.so) for the meshes of vox_meshes() below at preferred resolutions 7, 31
  and 63, each on the cube the oracle's voxel_box gives;
* ref_kernels.npz (only with --kernels, on a machine with a GPU): the outputs of the reference's
  applyK_OTFA_kernel, computeSensitivity_kernel, trySensMultiplier_kernel and
  filterSensitivity_kernel (oracle/_ref/libref_kernels.so) on the seeded inputs of
  tests/golden/ref_inputs.py.

Run from the repository root:  python tests/golden/make_ref_fixtures.py [--kernels] [--out DIR]
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import reference  # noqa: E402
from ref_inputs import CASES, FILTER_RADIUS, OC, P, inputs  # noqa: E402

KE_PARAMS = [(1.0, 1e6, 0.4), (1.0, 1.0, 0.3), (0.5, 2e5, 0.25)]


def stop_sequences():
    """Objective / constraint sequences for the stop test: converging geometric tails, noisy
    plateaus, a zero constraint (0 / 0 changes), a shrinking volume goal, and sequences of 1-3
    values (changes not yet defined)."""
    rng = np.random.default_rng(11)
    seqs = []
    for case in range(12):
        n = int(rng.integers(1, 40))
        c = 10.0 * (1 + rng.uniform(0.05, 0.5) * rng.uniform(0.3, 0.95) ** np.arange(n))
        if case % 3 == 1:
            c = c * (1 + rng.normal(0, 10 ** rng.uniform(-4, -2), n))
        g = np.zeros(n) if case % 4 == 0 else -0.4 * 0.02 * np.ones(n)
        if case % 4 == 3:
            g = 0.4 * (0.98 ** np.arange(1, n + 1) - 1)
        seqs.append((c, g))
    for n in (1, 2, 3):
        seqs.append((np.linspace(5, 4, n), np.zeros(n)))
    return seqs


def vox_meshes():
    """Closed meshes for the voxeliser pin (product mesh generators, deterministic)."""
    from robtop_b200 import configs

    s3 = configs.icosphere(3, radius=1.0)
    t = configs.torus(1.0, 0.35, 40, 20)
    return {
        "sphere": configs.icosphere(4, radius=1.0),
        "sphere_rotated": (configs.rigid_transform(s3[0], 11, (0.3, -0.2, 0.1)), s3[1]),
        "torus_rotated": (configs.rigid_transform(t[0], 12), t[1]),
        "box_half_voxel": configs.box_mesh((0.1, 0.1, 0.1), (0.9, 0.9, 0.9)),
        "box_flat": configs.box_mesh((0.0, 0.0, 0.0), (1.0, 0.37, 0.61)),
        "two_spheres": configs.merge_meshes(configs.icosphere(2, (0, 0, 0), 0.5),
                                            configs.icosphere(3, (1.3, 0.2, 0.1), 0.6)),
    }


VOX_PREFER = (7, 31, 63)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernels", action="store_true")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if os.path.exists(reference.KE_LIB):
        kes = np.stack([reference.template_matrix(h, E, nu) for h, E, nu in KE_PARAMS])
        np.savez_compressed(os.path.join(a.out, "ref_template_matrix.npz"), params=np.array(KE_PARAMS), ke=kes)
        print("template matrices written")
    if os.path.exists(reference.STOP_LIB):
        seqs = stop_sequences()
        flat = {}
        for i, (c, g) in enumerate(seqs):
            flat[f"c{i}"], flat[f"g{i}"] = c, g
            flat[f"stop{i}"] = reference.converge_run(1, 2, 5e-3, c, g)
            flat[f"stop_fabs{i}"] = reference.converge_run(1, 2, 5e-3, c, g, float_abs=True)
        np.savez_compressed(os.path.join(a.out, "ref_stop.npz"), n=len(seqs), **flat)
        print("stop-test results written")
    if os.path.exists(reference.VOX_LIB):
        import oracle as O

        out = {}
        for name, (v, f) in vox_meshes().items():
            for prefer in VOX_PREFER:
                R, bmin, bmax, _ = O.voxel_box(v, prefer)
                out[f"{name}/{prefer}"] = reference.voxelize_solid(v, f, R, bmin, bmax)
        np.savez_compressed(os.path.join(a.out, "ref_vox.npz"), **out)
        print("voxeliser bits written")
    if a.kernels:
        K = reference.Kernels()
        out = {}
        for name in CASES:
            cfg, KE, u, sens, eshell, ws = inputs(name)
            out[f"{name}/applyK"] = K.apply_k(cfg["eact"], cfg["vfix"] if ws else None, cfg["rho"], P, KE, u)
            out[f"{name}/sensitivity"] = K.sensitivity(cfg["eact"], cfg["rho"], P, KE, u)
            out[f"{name}/oc_try"] = K.oc_try(cfg["eact"], eshell, cfg["rho"], sens, OC["thres"], OC["step"],
                                             OC["damp"], OC["rhomin"])
            out[f"{name}/filter"] = K.filter(cfg["eact"], FILTER_RADIUS, sens)
        np.savez_compressed(os.path.join(a.out, "ref_kernels.npz"), **out)
        print("reference kernel outputs written:", sorted(out))


if __name__ == "__main__":
    main()
