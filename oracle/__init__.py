"""CPU oracle for the robtop solver hot path (TEST INFRASTRUCTURE ONLY).

A ctypes wrapper over ``oracle/liboracle.so`` (built from ``rt_oracle.c`` by
``oracle/Makefile``).  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference arm may import this package: it is the
checker, never the thing measured or shipped.

Parity status: "parity unpinned" — the reference cannot be compiled here and
ships no golden vectors; the restatement is pinned by the reference's own
known-answer tests (see ``tests/test_oracle_known_answers.py``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

SMOOTH_GS, SMOOTH_SGS, SMOOTH_JACOBI, SMOOTH_CHEBY = 0, 1, 2, 3
LMAX_STEPS = 30  # Lanczos steps of the Chebyshev bound estimate (the library uses the same count)


def build() -> str:
    """Compile the oracle library in place (gcc + OpenMP)."""
    srcs = [os.path.join(_HERE, f) for f in ("rt_oracle.c", "or_voxel.c", "rt_oracle.h")]
    if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < max(os.path.getmtime(s) for s in srcs):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


class Level(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ratio", C.c_int),
        ("eact", C.c_void_p), ("vact", C.c_void_p), ("vfix", C.c_void_p), ("w", C.c_void_p),
        ("st", C.c_void_p), ("u", C.c_void_p), ("f", C.c_void_p), ("r", C.c_void_p),
        ("ainv", C.c_void_p), ("aidx", C.c_void_p), ("na", C.c_int), ("lmax", C.c_double), ("d", C.c_void_p),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        sig = {
            "or_template_matrix": (None, [C.c_double, C.c_double, C.c_double, P]),
            "or_cube_vbits": (None, [C.c_int, P, P]),
            "or_cube_coarsen": (None, [C.c_int, P, P]),
            "or_bits_total": (C.c_long, [C.c_long, P]),
            "or_bitsat_rank": (None, [C.c_long, P, C.c_long, P, P]),
            "or_gs_maps": (None, [C.c_int, P, C.c_int, P, P, P]),
            "or_node_active": (None, [C.c_int, C.c_int, C.c_int, P, P]),
            "or_coarsen_elements": (None, [C.c_int, C.c_int, C.c_int, C.c_int, P, P]),
            "or_surface_nodes": (None, [C.c_int, C.c_int, C.c_int, P, P]),
            "or_penalty_weights": (None, [C.c_long, P, P, C.c_float, P]),
            "or_fine_applyK": (None, [P, P, P, P]),
            "or_fine_residual": (None, [P, P, P, P, P]),
            "or_fine_gs": (None, [P, P, P, P, C.c_int]),
            "or_fine_jacobi": (None, [P, P, P, P, C.c_double, P]),
            "or_st_applyA": (None, [P, P, P]),
            "or_st_residual": (None, [P, P, P, P]),
            "or_st_gs": (None, [P, P, P, C.c_int]),
            "or_st_jacobi": (None, [P, P, P, C.c_double, P]),
            "or_restrict": (None, [P, P, P, P]),
            "or_prolong_add": (None, [P, P, P, P]),
            "or_galerkin_from_elements": (None, [P, P, P, C.c_int]),
            "or_galerkin_from_stencil": (None, [P, P]),
            "or_coarsest_setup": (C.c_int, [P, C.c_int]),
            "or_coarsest_solve": (None, [P]),
            "or_vcycle": (C.c_double, [P, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int]),
            "or_pcg": (C.c_int, [P, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_double, P, P, C.c_double,
                                 C.c_int, P, P]),
            "or_dot": (C.c_double, [C.c_long, P, P]),
            "or_rng_uniform": (None, [C.c_uint64, C.c_long, P]),
            "or_rigid_basis": (C.c_int, [C.c_int, P, P, C.c_int, P]),
            "or_force_project": (None, [C.c_long, C.c_int, P, P, C.c_int, C.c_int, P, P]),
            "or_rigid_nodes": (None, [P, P]),
            "or_displacement_project": (None, [C.c_long, P, P]),
            "or_modified_pm": (C.c_double, [P, C.c_int, P, C.c_int, P, P, C.c_int, C.c_int, P, P, C.c_uint64,
                                            C.c_int, P, P]),
            "or_lanczos": (C.c_int, [P, C.c_int, P, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, P, P,
                                     C.c_int, C.c_int, P, C.c_uint64, C.c_int, C.c_double, C.c_int, P, P, P]),
            "or_tridiag_max_eig": (C.c_double, [C.c_int, P, P]),
            "or_cheby_coef": (None, [C.c_double, C.c_int, P, P]),
            "or_fine_cheby": (None, [P, P, P, P, P, P, C.c_int]),
            "or_st_cheby": (None, [P, P, P, P, P, C.c_int]),
            "or_lambda_max": (C.c_double, [P, C.c_int, P, C.c_uint64, C.c_int, P]),
            "or_sensitivity": (None, [C.c_int, C.c_int, C.c_int, P, P, C.c_float, P, P, P]),
            "or_filter": (None, [C.c_int, C.c_int, C.c_int, P, C.c_float, P, P]),
            "or_oc_try": (None, [C.c_long, P, P, P, P, C.c_float, C.c_float, C.c_float, C.c_float, P]),
            "or_oc_update": (C.c_float, [C.c_long, P, P, P, P, C.c_float, C.c_float, C.c_float, C.c_float,
                                         C.c_long, P, P]),
            "or_voxel_box": (None, [P, C.c_long, C.c_int, P, P, P, P]),
            "or_voxelize_solid": (None, [P, P, C.c_long, C.c_int, P, P, P]),
            "or_word_reverse": (None, [C.c_long, P]),
            "or_mma_init": (None, [C.c_long, P, P, P, P, P, P, P, P]),
            "or_mma_update": (C.c_double, [C.c_long, P, P, C.c_double, P, P, P, P, P, P, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data


# ----------------------------------------------------------------------------
# element template / occupancy
# ----------------------------------------------------------------------------
def template_matrix(E=1.0, nu=0.3, h=1.0):
    KE = np.zeros((24, 24), np.float64)
    lib().or_template_matrix(E, nu, h, ptr(KE))
    return KE


def cube_vbits(R, ebits):
    nw = ((R + 1) ** 3 + 31) // 32
    vb = np.zeros(nw, np.uint32)
    lib().or_cube_vbits(R, ptr(np.ascontiguousarray(ebits, np.uint32)), ptr(vb))
    return vb


def cube_coarsen(Rf, ebits):
    Rc = Rf // 2
    ec = np.zeros((Rc ** 3 + 31) // 32, np.uint32)
    lib().or_cube_coarsen(Rf, ptr(np.ascontiguousarray(ebits, np.uint32)), ptr(ec))
    return ec


def bits_total(bits):
    bits = np.ascontiguousarray(bits, np.uint32)
    return lib().or_bits_total(bits.size, ptr(bits))


def bitsat_rank(bits, q):
    bits = np.ascontiguousarray(bits, np.uint32)
    q = np.ascontiguousarray(q, np.int64)
    out = np.zeros(q.size, np.int32)
    lib().or_bitsat_rank(bits.size, ptr(bits), q.size, ptr(q), ptr(out))
    return out


def cube_hierarchy(R, ebits):
    """Per-level (R, ebits, vbits) of the reference's cubic bit hierarchy
    (grid/Grid.cpp:455-505): coarsen while more than 400 elements are solid."""
    levels = [(R, np.asarray(ebits, np.uint32), cube_vbits(R, ebits))]
    while bits_total(levels[-1][1]) > 400:
        Rf, ef, _ = levels[-1]
        ec = cube_coarsen(Rf, ef)
        levels.append((Rf // 2, ec, cube_vbits(Rf // 2, ec)))
    return levels


def gs_maps(vreso, vbits):
    nact = bits_total(vbits)
    vl = np.zeros(max(nact, 1), np.int32)
    gs_num = np.zeros(8, np.int32)
    nvgs = np.zeros(1, np.int32)
    lib().or_gs_maps(vreso, ptr(np.ascontiguousarray(vbits, np.uint32)), nact, ptr(vl), ptr(gs_num), ptr(nvgs))
    return vl[:nact], gs_num, int(nvgs[0])


# ----------------------------------------------------------------------------
# dense-box hierarchy
# ----------------------------------------------------------------------------
def node_active(eact):
    nz, ny, nx = eact.shape
    v = np.zeros((nz + 1, ny + 1, nx + 1), np.uint8)
    lib().or_node_active(nx, ny, nz, ptr(np.ascontiguousarray(eact, np.uint8)), ptr(v))
    return v


def coarsen_elements(eact, ratio):
    nz, ny, nx = eact.shape
    c = np.zeros(((nz + ratio - 1) // ratio, (ny + ratio - 1) // ratio, (nx + ratio - 1) // ratio), np.uint8)
    lib().or_coarsen_elements(nx, ny, nz, ratio, ptr(np.ascontiguousarray(eact, np.uint8)), ptr(c))
    return c


def surface_nodes(eact):
    nz, ny, nx = eact.shape
    s = np.zeros((nz + 1, ny + 1, nx + 1), np.uint8)
    lib().or_surface_nodes(nx, ny, nz, ptr(np.ascontiguousarray(eact, np.uint8)), ptr(s))
    return s


def level_plan(eact, skip=True):
    """Element activity of each real level and its coarsening ratio.  Mirrors the
    reference: halve while more than 400 elements are solid; with ``skip`` the
    first halving is a dummy level so the first coarse level is 4x coarser."""
    chain = [np.ascontiguousarray(eact, np.uint8)]
    while int(chain[-1].sum()) > 400:
        chain.append(coarsen_elements(chain[-1], 2))
    if skip and len(chain) >= 3:
        idx = [0] + list(range(2, len(chain)))
        ratios = [0, 4] + [2] * (len(chain) - 3)
    else:
        idx = list(range(len(chain)))
        ratios = [0] + [2] * (len(chain) - 1)
    return [chain[i] for i in idx], ratios


class Hierarchy:
    """Owns numpy arrays for every level and the ctypes Level descriptors."""

    def __init__(self, eact, rho, vfix=None, p=3.0, E=1.0, nu=0.3, h=1.0, skip=True, no_support=None):
        self.KE = template_matrix(E, nu, h)
        acts, ratios = level_plan(eact, skip)
        if len(acts) < 2:
            raise ValueError("grid too small for multigrid (<= 400 solid elements)")
        self.p = float(p)
        self.levels = []
        self.arrs = []
        self.no_support = (vfix is None or not np.any(vfix)) if no_support is None else no_support
        for i, (ea, ra) in enumerate(zip(acts, ratios)):
            nz, ny, nx = ea.shape
            nv = (nx + 1) * (ny + 1) * (nz + 1)
            d = {"eact": np.ascontiguousarray(ea, np.uint8), "vact": node_active(ea).ravel()}
            d["u"] = np.zeros(3 * nv)
            d["f"] = np.zeros(3 * nv)
            d["r"] = np.zeros(3 * nv)
            d["d"] = np.zeros(3 * nv)
            if i == 0:
                d["rho"] = np.ascontiguousarray(rho, np.float32).ravel().copy()
                d["w"] = np.zeros(nx * ny * nz)
                d["vfix"] = None if vfix is None else np.ascontiguousarray(vfix, np.uint8).ravel()
            else:
                d["st"] = np.zeros(243 * nv)
            L = Level()
            L.nx, L.ny, L.nz, L.ratio = nx, ny, nz, ra
            self.levels.append(L)
            self.arrs.append(d)
        last = self.arrs[-1]
        nact = int(last["vact"].sum())
        last["aidx"] = np.zeros(max(nact, 1), np.int32)
        last["ainv"] = np.zeros((3 * nact) ** 2)
        self._bind()
        self.LA = (Level * len(self.levels))(*self.levels)
        self.update_weights()

    def _bind(self):
        for L, d in zip(self.levels, self.arrs):
            L.eact = ptr(d["eact"])
            L.vact = ptr(d["vact"])
            L.vfix = ptr(d.get("vfix"))
            L.w = ptr(d.get("w"))
            L.st = ptr(d.get("st"))
            L.u, L.f, L.r = ptr(d["u"]), ptr(d["f"]), ptr(d["r"])
            L.d = ptr(d["d"])
            L.ainv = ptr(d.get("ainv"))
            L.aidx = ptr(d.get("aidx"))

    def refresh(self):
        self.LA = (Level * len(self.levels))(*self.levels)

    @property
    def nlev(self):
        return len(self.levels)

    def lv(self, i):
        return C.byref(self.LA, i * C.sizeof(Level))

    def update_weights(self):
        d = self.arrs[0]
        if getattr(self, "_w_fixed", False):
            return
        lib().or_penalty_weights(d["w"].size, ptr(d["eact"]), ptr(d["rho"]), self.p, ptr(d["w"]))

    def set_lmax(self, values):
        """Chebyshev bounds per smoothed level (e.g. the device's estimates, for parity)."""
        for i, v in enumerate(values):
            self.LA[i].lmax = float(v)
        self._lmax_fixed = True

    def set_weights(self, w):
        """Use given element weights rho^p instead of this library's powf.  The
        reference evaluates powf in FP32; C and CUDA powf may differ by an ulp, so
        operator-level parity tests share one set of weights (checked separately)."""
        self.arrs[0]["w"][:] = np.asarray(w, np.float32).astype(np.float64).ravel() * self.arrs[0]["eact"].ravel()
        self._w_fixed = True

    def update_stencil(self):
        """HierarchyGrid::update_stencil (grid/Grid.cpp:2108-2119)."""
        self.update_weights()
        ws = 0 if self.no_support else 1
        for i in range(1, self.nlev):
            if i == 1:
                lib().or_galerkin_from_elements(self.lv(0), self.lv(1), ptr(self.KE), ws)
            else:
                lib().or_galerkin_from_stencil(self.lv(i - 1), self.lv(i))
        rc = lib().or_coarsest_setup(self.lv(self.nlev - 1), 1 if self.no_support else 0)
        if not getattr(self, "_lmax_fixed", False):
            for i in range(self.nlev - 1):
                work = np.zeros(6 * self.arrs[i]["u"].size)
                self.LA[i].lmax = lib().or_lambda_max(self.lv(i), 1 if i == 0 else 0, ptr(self.KE), 0x51AB + i,
                                                      LMAX_STEPS, ptr(work))
        if rc != 0:
            raise RuntimeError("coarsest factorisation failed")

    def vcycle(self, smoother=SMOOTH_GS, npre=1, npost=1, omega=0.6):
        return lib().or_vcycle(self.LA, self.nlev, ptr(self.KE), smoother, npre, npost, omega, 0)

    def pcg(self, b, x=None, tol=1e-6, maxit=200, smoother=SMOOTH_SGS, npre=1, npost=1, omega=0.6):
        nv = self.arrs[0]["u"].size // 3
        x = np.zeros(3 * nv) if x is None else np.ascontiguousarray(x, np.float64).copy()
        b = np.ascontiguousarray(b, np.float64)
        work = np.zeros(6 * 3 * nv)
        rr = np.zeros(1)
        it = lib().or_pcg(self.LA, self.nlev, ptr(self.KE), smoother, npre, npost, omega, ptr(x), ptr(b), tol,
                          maxit, ptr(rr), ptr(work))
        return x, it, float(rr[0])

    def applyK(self, u):
        out = np.zeros_like(u)
        lib().or_fine_applyK(self.lv(0), ptr(self.KE), ptr(np.ascontiguousarray(u)), ptr(out))
        return out


def rng_uniform(seed, n):
    out = np.zeros(n)
    lib().or_rng_uniform(seed, n, ptr(out))
    return out


def tridiag_max_eig(alpha, beta):
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.ascontiguousarray(beta, np.float64)
    return lib().or_tridiag_max_eig(a.size, ptr(a), ptr(b))


# ----------------------------------------------------------------------------
# solid mesh voxeliser (voxelizer/voxelize_main.cpp:290-402, cpu_voxelizer.cpp:194-322)
# ----------------------------------------------------------------------------
def voxel_box(coords, prefer_reso):
    """(reso, bmin, bmax, unit) of the padded power-of-two cube around the vertices."""
    coords = np.ascontiguousarray(coords, np.float32).reshape(-1)
    r = np.zeros(1, np.int32)
    bmin, bmax, unit = (np.zeros(3, np.float32) for _ in range(3))
    lib().or_voxel_box(ptr(coords), coords.size // 3, int(prefer_reso), ptr(r), ptr(bmin), ptr(bmax), ptr(unit))
    return int(r[0]), bmin, bmax, unit


def voxelize_solid(coords, tris, reso, bmin, unit):
    """Solid bits of the mesh, reso^3, bit x + y*reso + z*reso^2, most significant bit first."""
    coords = np.ascontiguousarray(coords, np.float32).reshape(-1)
    tris = np.ascontiguousarray(tris, np.int32).reshape(-1)
    bmin = np.ascontiguousarray(bmin, np.float32)
    unit = np.ascontiguousarray(unit, np.float32)
    bits = np.zeros((reso ** 3 + 31) // 32, np.uint32)
    lib().or_voxelize_solid(ptr(coords), ptr(tris), tris.size // 3, int(reso), ptr(bmin), ptr(unit), ptr(bits))
    return bits


def word_reverse(bits):
    out = np.array(bits, np.uint32, copy=True)
    lib().or_word_reverse(out.size, ptr(out))
    return out


class MMA:
    """The oracle's MMA state for one constraint (or_mma.c): bounds xmin, xmax (arrays or
    scalars); update(df, dg, g) takes one step and returns the multiplier."""

    def __init__(self, n, xmin, xmax):
        self.n = int(n)
        self.xmin = np.ascontiguousarray(np.broadcast_to(np.asarray(xmin, np.float64), (self.n,)))
        self.xmax = np.ascontiguousarray(np.broadcast_to(np.asarray(xmax, np.float64), (self.n,)))
        z = lambda: np.zeros(self.n)
        self.x, self.low, self.upp, self.alpha, self.beta, self.lastdx = z(), z(), z(), z(), z(), z()
        self.work = np.zeros(4 * self.n)
        self.dxnorm = 0.0
        lib().or_mma_init(self.n, ptr(self.xmin), ptr(self.xmax), ptr(self.x), ptr(self.low), ptr(self.upp),
                          ptr(self.alpha), ptr(self.beta), ptr(self.lastdx))

    def update(self, df, dg, g):
        df = np.ascontiguousarray(df, np.float64)
        dg = np.ascontiguousarray(dg, np.float64)
        dn = np.zeros(1)
        lam = lib().or_mma_update(self.n, ptr(df), ptr(dg), float(g), ptr(self.xmin), ptr(self.xmax), ptr(self.x),
                                  ptr(self.low), ptr(self.upp), ptr(self.alpha), ptr(self.beta), ptr(self.lastdx),
                                  ptr(dn), ptr(self.work))
        self.dxnorm = float(dn[0])
        return lam
