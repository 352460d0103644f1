"""The reference-signature C++ layer (robtop_compat.h), driven the way robtop.cpp and
TestSuit drive robtop, compared with the CPU oracle on the same problem."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from robtop_b200 import build as B
from robtop_b200 import configs

pytestmark = pytest.mark.gpu


def run_driver():
    exe = B.build_compat_driver()
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    vals = {}
    rigid = []
    for line in out.stdout.splitlines():
        if line.startswith("-- u_rigid"):
            rigid.append(float(line.split("=")[1]))
            continue
        if line.startswith("--"):
            continue
        k, v = line.split()
        vals[k] = float(v)
    return vals, rigid


def test_compat_flow_matches_oracle():
    vals, rigid = run_driver()
    cfg = configs.cantilever(24, 12, 12)
    assert vals["load_nodes"] == cfg["load_nodes"].size
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    H.update_stencil()
    assert vals["levels"] == H.nlev
    # test_rigid_displacement: K u_rigid vanishes away from the supports; with supports the
    # residual is nonzero only through the clamped nodes, so compare with the oracle's value
    # (six modes from the explicit call, six more from selfTest, which repeats it)
    assert len(rigid) == 12 and np.allclose(rigid[:6], rigid[6:], rtol=1e-9, atol=0)
    # solveFEM: V-cycles to 1e-4 on the preloaded force
    b = cfg["fload"].ravel().copy()
    H.arrs[0]["f"][:] = b
    H.arrs[0]["u"][:] = 0
    rel = 1
    while rel > 1e-4:
        rel = H.vcycle(O.SMOOTH_GS, 1, 1)
    c_or = b @ H.arrs[0]["u"]
    assert vals["rel_residual"] <= 1e-4
    assert abs(vals["compliance"] - c_or) <= 1e-4 * abs(c_or)
    # modifiedPM: worst-case compliance (random start differs in seed; the eigenvalue does not)
    assert vals["worst_compliance"] > 0
    x, _, _ = H.pcg(b / np.linalg.norm(b), tol=1e-10)
    assert vals["worst_compliance"] >= (b / np.linalg.norm(b)) @ x * (1 - 1e-3)
    assert abs(vals["volume"] - 0.4) <= 2e-4
    # buildGrids(coords, trifaces): the device voxeliser's solid cells = the oracle's
    v = np.array([0, 0, 0, 24, 0, 0, 24, 12, 0, 0, 12, 0, 0, 0, 12, 24, 0, 12, 24, 12, 12, 0, 12, 12], np.float32)
    f = np.array([0, 2, 1, 0, 3, 2, 4, 5, 6, 4, 6, 7, 0, 1, 5, 0, 5, 4, 2, 3, 7, 2, 7, 6, 0, 4, 7, 0, 7, 3, 1, 2, 6,
                  1, 6, 5], np.int32)
    R, bmin, bmax, unit = O.voxel_box(v, 31)
    assert vals["mesh_elements"] == O.bits_total(O.voxelize_solid(v, f, R, bmin, unit)) > 0
    assert vals["mesh_levels"] >= 2


def test_compat_remaining_entry_points():
    """The projection API (optimization/projection.h:16-65), Grid::elementCompliance,
    checkAdjointVariable, RayleighGradient, inCompleteModiPM, MGPSOR, selfTest and the density
    file round trip, driven through the reference-signature layer."""
    vals, rigid = run_driver()
    assert vals["adjoint_ok"] == 1 and vals["adjoint_zero_ok"] == 0
    # element compliances of the worst-case displacement sum to its u.K u (the modified power
    # method's last displacement is one V-cycle from the last load, so f.u differs from it)
    assert abs(vals["element_compliance_sum"] - vals["worst_uKu"]) <= 1e-5 * vals["worst_uKu"]
    cfg = configs.cantilever(24, 12, 12)
    assert vals["n_loadnodes"] == cfg["load_nodes"].size
    # wsff: the support force of the unit worst-case load has norm 1 and P keeps it
    assert abs(vals["support_norm2"] - 1.0) <= 1e-9
    assert abs(vals["pnorm"] - 1.0) <= 1e-9
    assert abs(vals["projected_norm2"] - 1.0) <= 1e-9
    assert abs(vals["restored_norm2"] - 1.0) <= 1e-9
    # at the worst-case displacement u = K^-1 f (|f| = 1): |P u|^2 / u.K u = lambda
    lam = vals["worst_compliance3"]
    assert abs(vals["rayleigh_pnorm"] / vals["rayleigh_knorm"] - lam) <= 1e-3 * lam
    # the incomplete power method reaches the worst case to within its 1e-2 force-change threshold
    assert 0.9 * lam <= vals["incomplete_pm"] <= lam * (1 + 1e-6)
    # MGPSOR (optimization/optimization.cpp:474-535) ends with u = x / |P x| and returns u.K u =
    # x.K x / |P x|^2, the reciprocal of the Rayleigh quotient it converged: 1 / lambda
    assert abs(vals["mgpsor"] * lam - 1.0) <= 1e-2
    assert vals["density_roundtrip"] == 1
    # optimization(): at most the 12 iterations asked for, the goal at the volume ratio, finite
    # compliances (the stop test needs at least four values before it can pass)
    assert 1 <= vals["opt_iterations"] <= 12
    assert vals["opt_iterations"] == 12 or vals["opt_iterations"] >= 6
    assert abs(vals["opt_last_volume_goal"] - 0.4) <= 1e-6
    assert 0 < vals["opt_first_compliance"] < 1e30 and 0 < vals["opt_last_compliance"] < 1e30
    # three MMA steps (MMA::mma_t, the testtest2011 loop) from the middle of the bounds (0.5005)
    # move the volume towards the 0.4 target
    assert 0 < vals["mma_compliance"] < 1e30
    assert 0.3 < vals["mma_volume"] < 0.5
