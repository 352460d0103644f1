"""The reference's own code, compiled from its sources (test infrastructure only).

``make -C oracle ref`` builds, from the reference tree (default /root/reference, present only
where the reference is mounted), these libraries into oracle/_ref/:

* libref_ke.so: element/templateMatrix.cpp:31-124 (initTemplateMatrix) on the host;
* libref_stop.so, libref_stop_fabs.so: snippet::converge_criteria (utils/snippet.h:156-213), the
  optimisation loop's stop test, on the host, with g++'s integer abs() of the change and with the
  floating-point one;
* libref_vox.so: cpu_voxelizer::cpu_voxelize_mesh_solid (voxelizer/cpu_voxelizer.cpp:262-322),
  the solid mesh voxeliser, on the host, against GLM / trimesh2 stand-ins;
* libref_kernels.so: applyK_OTFA_kernel (grid/Grid.cu:2439-2517), computeSensitivity_kernel and
  trySensMultiplier_kernel (optimization/optimization.cu:44-162) and filterSensitivity_kernel
  (grid/Grid.cu:2323-2409) for sm_100a, driven on dense element boxes (needs a GPU to run).

The built files travel with the repository to GPU machines; the sources do not.  Nothing on the
product path loads these libraries: the tests use them to pin the oracle and the CUDA path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
KE_LIB = os.path.join(REF_DIR, "libref_ke.so")
KERNELS_LIB = os.path.join(REF_DIR, "libref_kernels.so")
STOP_LIB = os.path.join(REF_DIR, "libref_stop.so")
STOP_FABS_LIB = os.path.join(REF_DIR, "libref_stop_fabs.so")
VOX_LIB = os.path.join(REF_DIR, "libref_vox.so")
REFERENCE_TREE = os.environ.get("ROBTOP_REFERENCE", "/root/reference")


def build() -> bool:
    """Build oracle/_ref/ when the reference tree is present; True if both libraries exist."""
    if os.path.isdir(REFERENCE_TREE):
        subprocess.check_call(["make", "-s", "-C", _HERE, "ref", f"REF={REFERENCE_TREE}"])
    return os.path.exists(KE_LIB) and os.path.exists(KERNELS_LIB)


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def template_matrix(h=1.0, E=1.0, nu=0.3):
    """KE (24x24) from the reference's initTemplateMatrix."""
    L = C.CDLL(KE_LIB)
    L.ref_template_matrix.argtypes = [C.c_double, C.c_double, C.c_double, C.c_void_p]
    out = np.zeros(576)
    L.ref_template_matrix(h, E, nu, _p(out))
    return out.reshape(24, 24)


def converge_run(n_constrain, max_counter, thres, values, constraints, float_abs=False):
    """The reference's converge_criteria(n_constrain, max_counter, thres) fed the objective values
    and the constraint rows in order; returns its update() results (1 = stop).  ``float_abs``
    selects the build in which abs() of the change is the floating-point one (the header under
    MSVC) instead of g++'s integer abs."""
    L = C.CDLL(STOP_FABS_LIB if float_abs else STOP_LIB)
    L.ref_converge_run.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    v = np.ascontiguousarray(values, np.float64)
    g = np.ascontiguousarray(np.reshape(constraints, (v.size, n_constrain)), np.float64)
    out = np.zeros(v.size, np.int32)
    L.ref_converge_run(n_constrain, max_counter, thres, v.size, _p(v), _p(g), _p(out))
    return out


def voxelize_solid(coords, tris, reso, bmin, bmax):
    """The reference's CPU solid voxeliser (cpu_voxelizer::cpu_voxelize_mesh_solid) on the cube
    [bmin, bmax] at reso^3: bits x + y reso + z reso^2, most significant bit first."""
    L = C.CDLL(VOX_LIB)
    P = C.c_void_p
    L.ref_voxelize_solid.argtypes = [P, C.c_long, P, C.c_long, P, P, C.c_int, P]
    v = np.ascontiguousarray(coords, np.float32).reshape(-1, 3)
    f = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    lo = np.ascontiguousarray(bmin, np.float32)
    hi = np.ascontiguousarray(bmax, np.float32)
    bits = np.zeros((reso ** 3 + 31) // 32, np.uint32)
    L.ref_voxelize_solid(_p(v), v.shape[0], _p(f), f.shape[0], _p(lo), _p(hi), int(reso), _p(bits))
    return bits


class Kernels:
    """The reference's CUDA kernels on a dense element box (arrays in the library's dense layout:
    elements x fastest over (nz, ny, nx), node vectors [3][(nx+1)(ny+1)(nz+1)])."""

    def __init__(self):
        L = C.CDLL(KERNELS_LIB)
        P, I, F = C.c_void_p, C.c_int, C.c_float
        L.ref_apply_k.argtypes = [I, I, I, P, P, P, F, P, P, P]
        L.ref_sensitivity.argtypes = [I, I, I, P, P, F, P, P, P]
        L.ref_oc_try.argtypes = [I, I, I, P, P, P, P, F, F, F, F, P]
        L.ref_filter.argtypes = [I, I, I, P, F, P, P]
        self.L = L

    @staticmethod
    def _box(eact):
        e = np.ascontiguousarray(eact, np.uint8)
        nz, ny, nx = e.shape
        return e, nx, ny, nz

    def apply_k(self, eact, vfix, rho, p, KE, u):
        e, nx, ny, nz = self._box(eact)
        nv = (nx + 1) * (ny + 1) * (nz + 1)
        f = np.zeros(3 * nv)
        vf = None if vfix is None else np.ascontiguousarray(vfix, np.uint8).ravel()
        st = self.L.ref_apply_k(nx, ny, nz, _p(e), _p(vf), _p(np.ascontiguousarray(rho, np.float32).ravel()), p,
                                _p(np.ascontiguousarray(KE, np.float64).ravel()),
                                _p(np.ascontiguousarray(u, np.float64)), _p(f))
        assert st == 0
        return f

    def sensitivity(self, eact, rho, p, KE, u):
        e, nx, ny, nz = self._box(eact)
        s = np.zeros(nx * ny * nz, np.float32)
        st = self.L.ref_sensitivity(nx, ny, nz, _p(e), _p(np.ascontiguousarray(rho, np.float32).ravel()), p,
                                    _p(np.ascontiguousarray(KE, np.float64).ravel()),
                                    _p(np.ascontiguousarray(u, np.float64)), _p(s))
        assert st == 0
        return s

    def oc_try(self, eact, eshell, rho, sens, thres, step, damp, rhomin):
        e, nx, ny, nz = self._box(eact)
        out = np.zeros(nx * ny * nz, np.float32)
        sh = None if eshell is None else np.ascontiguousarray(eshell, np.uint8).ravel()
        st = self.L.ref_oc_try(nx, ny, nz, _p(e), _p(sh), _p(np.ascontiguousarray(rho, np.float32).ravel()),
                               _p(np.ascontiguousarray(sens, np.float32).ravel()), thres, step, damp, rhomin, _p(out))
        assert st == 0
        return out

    def filter(self, eact, radius, sens):
        e, nx, ny, nz = self._box(eact)
        out = np.zeros(nx * ny * nz, np.float32)
        st = self.L.ref_filter(nx, ny, nz, _p(e), radius, _p(np.ascontiguousarray(sens, np.float32).ravel()), _p(out))
        assert st == 0
        return out
