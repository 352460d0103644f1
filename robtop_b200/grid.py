"""Host-side mirror of robtop's ``grid::HierarchyGrid`` / ``grid::Grid`` API.

Same method names and argument meaning as ``grid/Grid.h:172-692`` of the
reference; every call goes through the C ABI in ``librtb200.so``.  Vectors are
exchanged as numpy arrays in the dense layout (SoA ``[3][nv]``, x fastest) or,
with ``layout=LAYOUT_REF_GS``, in the reference's GS-colour-ordered padded
layout (``grid/Grid.cpp:2045-2106``).  Errors raise ``RTError`` instead of the
reference's print-and-continue / ``exit(-1)``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A
from ._capi import check


def _dp(t):
    """Device pointer of a torch CUDA tensor (plumbing only).  The library runs on its context's
    own stream, so torch's pending work on the tensor (the copy or fill that made it) is waited
    for first."""
    import torch

    torch.cuda.current_stream(t.device).synchronize()
    return C.c_void_p(t.data_ptr())


def _p(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class Context:
    """One device + one CUDA stream (``stream`` may be a caller's cudaStream_t handle)."""

    def __init__(self, device=0, stream=None):
        self._h = C.c_void_p()
        self.device = int(device)
        check(A.lib().rt_ctx_create(device, stream, C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def sync(self):
        check(A.lib().rt_ctx_sync(self._h), self._h)

    def last_error(self):
        return A.lib().rt_last_error(self._h).decode()

    def launches(self):
        return int(A.lib().rt_launch_count(self._h))

    def profile(self, on=True):
        check(A.lib().rt_profile_enable(self._h, 1 if on else 0), self._h)

    def profile_reset(self):
        check(A.lib().rt_profile_reset(self._h), self._h)

    def profile_stats(self):
        out = {}
        i = 0
        name = C.create_string_buffer(128)
        n = C.c_longlong()
        ms = C.c_double()
        while A.lib().rt_profile_query(self._h, i, name, 128, C.byref(n), C.byref(ms)) == A.RT_OK:
            out[name.value.decode()] = (int(n.value), float(ms.value))
            i += 1
        return out

    def close(self):
        if self._h:
            A.lib().rt_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_params(**kw):
    p = A.Params()
    A.lib().rt_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


class Grid:
    """One level of the hierarchy (``grid::Grid``, grid/Grid.h:172-532)."""

    def __init__(self, hier, level):
        self._H = hier
        self._layer = level
        info = A.LevelInfo()
        check(A.lib().rt_hier_level_info(hier.handle, level, C.byref(info)), hier.ctx.handle)
        self.nx, self.ny, self.nz, self.ratio = info.nx, info.ny, info.nz, info.ratio
        self.n_box_nodes = int(info.n_nodes)
        self.n_vertices = int(info.n_active_nodes)
        self.n_elements = int(info.n_active_elements)

    # sizes ---------------------------------------------------------------
    @property
    def nv(self):
        return self.n_box_nodes

    @property
    def ne(self):
        return self.nx * self.ny * self.nz

    def n_nodes(self):
        return self.n_vertices

    def n_valid_elements(self):
        return self.n_elements

    # operators (grid/Grid.cu) --------------------------------------------
    def update_residual(self):
        self._H._c(A.lib().rt_update_residual(self._H.handle, self._layer))

    def gs_relax(self, n_times=1):
        self._H._c(A.lib().rt_smooth(self._H.handle, self._layer, A.SMOOTH_GS, n_times, 1.0))

    def smooth(self, smoother, sweeps=1, omega=0.6):
        self._H._c(A.lib().rt_smooth(self._H.handle, self._layer, smoother, sweeps, omega))

    def restrict_residual(self):
        self._H._c(A.lib().rt_restrict_residual(self._H.handle, self._layer))

    def prolongate_correction(self):
        self._H._c(A.lib().rt_prolongate_correction(self._H.handle, self._layer))

    def solve_fem_host(self):
        """Coarsest direct solve (on the device, despite the reference's name)."""
        self._H._c(A.lib().rt_coarsest_solve(self._H.handle))

    def applyK(self, u):
        assert self._layer == 0
        u = np.ascontiguousarray(u, np.float64)
        out = np.zeros_like(u)
        self._H._c(A.lib().rt_apply_K(self._H.handle, _p(u), _p(out)))
        return out

    def compliance(self):
        c = C.c_double()
        self._H._c(A.lib().rt_compliance(self._H.handle, C.byref(c)))
        return c.value

    def relative_residual(self):
        c = C.c_double()
        self._H._c(A.lib().rt_relative_residual(self._H.handle, C.byref(c)))
        return c.value

    def filterSensitivity(self, radii):
        self._H._c(A.lib().rt_filter_sensitivity(self._H.handle, float(radii)))

    def init_rho(self, rh0):
        self._H._c(A.lib().rt_init_density(self._H.handle, float(rh0)))

    # fields ---------------------------------------------------------------
    def _get(self, field, layout, shape, dtype):
        out = np.zeros(shape, dtype)
        self._H._c(A.lib().rt_get(self._H.handle, field, self._layer, layout, _p(out)))
        return out

    def _put(self, field, layout, arr, dtype):
        arr = np.ascontiguousarray(arr, dtype)
        self._H._c(A.lib().rt_put(self._H.handle, field, self._layer, layout, _p(arr)))

    def ref_gs_map(self):
        vm = np.zeros(self.nv, np.int32)
        ngs = C.c_int()
        gsn = np.zeros(8, np.int32)
        self._H._c(A.lib().rt_ref_gs_map(self._H.handle, self._layer, _p(vm), C.byref(ngs), _p(gsn)))
        return vm, int(ngs.value), gsn

    def _vec_shape(self, layout):
        if layout == A.LAYOUT_REF_GS:
            return 3 * self.ref_gs_map()[1]
        return 3 * self.nv

    def getDisplacement(self, layout=A.LAYOUT_DENSE):
        return self._get(A.FIELD_U, layout, self._vec_shape(layout), np.float64)

    def getForce(self, layout=A.LAYOUT_DENSE):
        return self._get(A.FIELD_F, layout, self._vec_shape(layout), np.float64)

    def getResidual(self, layout=A.LAYOUT_DENSE):
        return self._get(A.FIELD_R, layout, self._vec_shape(layout), np.float64)

    def setDisplacement(self, u, layout=A.LAYOUT_DENSE):
        self._put(A.FIELD_U, layout, u, np.float64)

    def setForce(self, f, layout=A.LAYOUT_DENSE):
        self._put(A.FIELD_F, layout, f, np.float64)

    def setResidual(self, r, layout=A.LAYOUT_DENSE):
        self._put(A.FIELD_R, layout, r, np.float64)

    def getRho(self):
        return self._get(A.FIELD_RHO, A.LAYOUT_DENSE, self.ne, np.float32)

    def setRho(self, rho):
        self._put(A.FIELD_RHO, A.LAYOUT_DENSE, rho, np.float32)

    def getPenalty(self):
        """Element weights powf(rho, p) used by the operator (refreshed by update_stencil)."""
        return self._get(A.FIELD_PENALTY, A.LAYOUT_DENSE, self.ne, np.float32)

    def getSens(self):
        return self._get(A.FIELD_SENS, A.LAYOUT_DENSE, self.ne, np.float32)

    def setSens(self, s):
        self._put(A.FIELD_SENS, A.LAYOUT_DENSE, s, np.float32)

    def getStencil(self):
        return self._get(A.FIELD_STENCIL, A.LAYOUT_DENSE, 243 * self.nv, np.float64)

    def setStencil(self, st):
        self._put(A.FIELD_STENCIL, A.LAYOUT_DENSE, st, np.float64)

    def getVact(self):
        return self._get(A.FIELD_VACT, A.LAYOUT_DENSE, self.nv, np.uint8)

    def getEact(self):
        return self._get(A.FIELD_EACT, A.LAYOUT_DENSE, self.ne, np.uint8)

    def elementCompliance(self, u):
        """Grid::elementCompliance (grid/Grid.cu:3434-3480): rho_e^p u_e.KE u_e per element (dense
        element order) for the level-0 displacement u."""
        assert self._layer == 0
        import torch

        ud = torch.as_tensor(np.ascontiguousarray(u, np.float64), device=f"cuda:{self._H.ctx.device}")
        ce = torch.zeros(self.ne, dtype=torch.float32, device=ud.device)
        self._H._c(A.lib().rt_element_compliance(self._H.handle, _dp(ud), _dp(ce)))
        self._H.ctx.sync()
        return ce.cpu().numpy()

    def reset_displacement(self):
        self.setDisplacement(np.zeros(3 * self.nv))

    def reset_force(self):
        self.setForce(np.zeros(3 * self.nv))

    def reset_residual(self):
        self.setResidual(np.zeros(3 * self.nv))


class HierarchyGrid:
    """``grid::HierarchyGrid`` (grid/Grid.h:534-692) on the device."""

    def __init__(self, ctx: Context, params=None):
        self.ctx = ctx
        self.params = params if params is not None else default_params()
        self._h = C.c_void_p()
        self._grids = []
        self._children = []

    @property
    def handle(self):
        return self._h

    def _c(self, status):
        return check(status, self.ctx.handle)

    # construction (grid/Grid.cpp:455-712) --------------------------------
    def genFromMesh(self, solid_bit, out_reso):
        """Cubic ``out_reso[0]^3`` bit grid (LSB-first words, bit x + y R + z R^2)."""
        reso = int(out_reso[0]) if np.ndim(out_reso) else int(out_reso)
        bits = np.ascontiguousarray(solid_bit, np.uint32)
        self._c(A.lib().rt_hier_create_from_bits(self.ctx.handle, C.byref(self.params), reso, _p(bits),
                                                 C.byref(self._h)))
        self._init_levels()

    def genFromTriMesh(self, pcoords, facevertices, prefer_reso):
        """HierarchyGrid::genFromMesh(pcoords, facevertices) (grid/Grid.cpp:184-205): solid
        voxelisation of the closed triangle mesh on the device, then the hierarchy."""
        v = np.ascontiguousarray(pcoords, np.float32).reshape(-1)
        f = np.ascontiguousarray(facevertices, np.int32).reshape(-1)
        self._c(A.lib().rt_hier_create_from_mesh(self.ctx.handle, C.byref(self.params), _p(v), v.size // 3, _p(f),
                                                 f.size // 3, int(prefer_reso), C.byref(self._h)))
        self._init_levels()

    def genFromBox(self, eact):
        """Dense element-activity box ``eact[nz, ny, nx]`` (x fastest)."""
        eact = np.ascontiguousarray(eact, np.uint8)
        nz, ny, nx = eact.shape
        self._c(A.lib().rt_hier_create(self.ctx.handle, C.byref(self.params), nx, ny, nz, _p(eact),
                                       C.byref(self._h)))
        self._init_levels()

    def _init_levels(self):
        n = A.lib().rt_hier_n_levels(self._h)
        self._grids = [Grid(self, i) for i in range(n)]

    def __getitem__(self, i):
        return self._grids[i]

    def n_grid(self):
        return len(self._grids)

    def setMode(self, mode):
        self.params.mode = mode
        self.set_params(self.params)

    def set_params(self, params):
        self.params = params
        self._c(A.lib().rt_hier_set_params(self._h, C.byref(params)))

    def isForceFree(self):
        return self.params.mode in (A.MODE_NSFF, A.MODE_WSFF)

    def hasSupport(self):
        return self.params.mode in (A.MODE_WSCF, A.MODE_WSFF)

    def template_matrix(self):
        KE = np.zeros((24, 24))
        self._c(A.lib().rt_template_matrix(self._h, _p(KE)))
        return KE

    # boundary conditions ---------------------------------------------------
    def surface_nodes(self):
        s = np.zeros(self[0].nv, np.uint8)
        self._c(A.lib().rt_surface_nodes(self._h, _p(s)))
        return s

    def set_support(self, vfix):
        vfix = np.ascontiguousarray(vfix, np.uint8).ravel()
        self._c(A.lib().rt_set_support(self._h, _p(vfix)))

    def set_shell(self, eshell):
        """Shell elements (dense level-0 order) whose density the OC update holds at 1; None clears."""
        if eshell is None:
            self._c(A.lib().rt_set_shell(self._h, None))
            return
        e = np.ascontiguousarray(eshell, np.uint8)
        self._c(A.lib().rt_set_shell(self._h, _p(e)))

    def set_load_nodes(self, nodes, normals):
        nodes = np.ascontiguousarray(nodes, np.int32)
        normals = np.ascontiguousarray(normals, np.float64).reshape(-1)
        self._c(A.lib().rt_set_load_nodes(self._h, int(nodes.size), _p(nodes), _p(normals)))

    # multigrid -----------------------------------------------------------------
    def update_stencil(self):
        self._c(A.lib().rt_update_stencil(self._h))

    def autotune(self, reps=5):
        """Choose the finest-level kernel launch shapes (rt_autotune); returns them per kernel."""
        self._c(A.lib().rt_autotune(self._h, reps))
        return self.tuning()

    def set_tiles(self, variant, rows, zchunk):
        """One launch shape for every finest-level kernel of both precisions (rt_set_tuning);
        returns the shapes as tuning() reports them."""
        for prec in (A.FP32, A.FP64):
            for m in range(4):
                self._c(A.lib().rt_set_tuning(self._h, prec, m, variant, rows, zchunk))
        return self.tuning()

    def tuning(self):
        """The current launch shapes (and, after autotune, their measured times) per kernel."""
        out = {}
        names = ["residual", "applyK", "jacobi", "chebyshev"]
        for prec, pname in ((A.FP32, "f32"), (A.FP64, "f64")):
            for m, mname in enumerate(names):
                v, ty, zc, us = C.c_int(), C.c_int(), C.c_int(), C.c_double()
                self._c(A.lib().rt_tuning_info(self._h, prec, m, C.byref(v), C.byref(ty), C.byref(zc), C.byref(us)))
                out[f"{mname}_{pname}"] = {"variant": ["smem_tile", "register_march", "register_march_prefetch", "smem_tile_pipelined", "smem_tile_pairs_f32",
                                                       "sum_factorised", "smem_tile_pipelined_tma",
                                                       "smem_tile_pipelined_tma_x31"][v.value], "rows": ty.value,
                                           "zchunk": zc.value, "us": round(us.value, 2)}
        for lvl in range(1, self.n_grid() - 1):
            on, t0, t1 = C.c_int(), C.c_double(), C.c_double()
            if A.lib().rt_level_fused_info(self._h, lvl, C.byref(on), C.byref(t0), C.byref(t1)) == A.RT_OK:
                out[f"chebyshev_f32_level{lvl}"] = {"fused": bool(on.value),
                                                    "us_8_steps": {"separate": round(t0.value, 2),
                                                                   "fused": round(t1.value, 2)}}
        for st, sname in ((0, "f32"), (1, "bf16")):
            v, u0, u1 = C.c_int(), C.c_double(), C.c_double()
            self._c(A.lib().rt_level_kernel_info(self._h, st, C.byref(v), C.byref(u0), C.byref(u1)))
            if u0.value > 0:
                out[f"stencil_chebyshev_{sname}"] = {"variant": ["lane_split", "bulk_copy"][v.value],
                                                     "us": {"lane_split": round(u0.value, 2),
                                                            "bulk_copy": round(u1.value, 2)}}
        return out

    def smoother_lmax(self, level):
        v = C.c_double()
        self._c(A.lib().rt_smoother_lmax(self._h, level, C.byref(v)))
        return v.value

    def v_cycle(self, pre_relax=1, post_relax=1):
        r = C.c_double()
        self._c(A.lib().rt_vcycle(self._h, pre_relax, post_relax, C.byref(r)))
        return r.value

    def pcg(self, tol=1e-6, maxit=200):
        info = A.SolveInfo()
        st = A.lib().rt_pcg(self._h, tol, maxit, C.byref(info))
        if st not in (A.RT_OK, A.RT_ENOCONV):
            self._c(st)
        return info

    def worst_case(self, method=A.WORST_LANCZOS, k=16, inner_tol=1e-8, seed=0):
        lam = C.c_double()
        info = A.SolveInfo()
        self._c(A.lib().rt_worst_case(self._h, method, k, inner_tol, seed, C.byref(lam), C.byref(info)))
        return lam.value, info

    def worst_case_block(self, block_size=8, n_blocks=2, inner_tol=1e-8, seed=0):
        """Block Lanczos (rt_worst_case_block): each block step's inner solves run as one graph."""
        lam = C.c_double()
        info = A.SolveInfo()
        self._c(A.lib().rt_worst_case_block(self._h, block_size, n_blocks, inner_tol, seed, C.byref(lam),
                                            C.byref(info)))
        return lam.value, info

    # projection API (optimization/projection.h:16-65) ---------------------------------------
    def _dev(self, a, dtype=np.float64):
        import torch

        return torch.as_tensor(np.ascontiguousarray(a, dtype), device=f"cuda:{self.ctx.device}")

    def getLoadNodes(self):
        """getLoadNodes (optimization/projection.cpp:129-143): dense level-0 ids, increasing."""
        n = C.c_int()
        self._c(A.lib().rt_load_nodes(self._h, C.byref(n), None))
        ids = np.zeros(n.value, np.int32)
        self._c(A.lib().rt_load_nodes(self._h, C.byref(n), _p(ids)))
        return ids

    def forceProject(self, f):
        """forceProject (optimization/projection.cu:165-231): P f for a dense [3][nv] force."""
        fd = self._dev(f)
        self._c(A.lib().rt_force_project(self._h, _dp(fd)))
        self.ctx.sync()
        return fd.cpu().numpy()

    def getForceSupport(self, f):
        """getForceSupport (optimization/projection.cu:307-338): the load-node values, [3][nload]."""
        fd = self._dev(f)
        n = self.getLoadNodes().size
        import torch

        fs = torch.zeros(3 * n, dtype=torch.float64, device=fd.device)
        self._c(A.lib().rt_get_force_support(self._h, _dp(fd), _dp(fs)))
        self.ctx.sync()
        return fs.cpu().numpy().reshape(3, n)

    def setForceSupport(self, fs):
        """setForceSupport (optimization/projection.cu:340-369): a dense force that is fs on the load
        nodes and zero elsewhere."""
        import torch

        fsd = self._dev(np.asarray(fs).reshape(-1))
        f = torch.zeros(3 * self[0].nv, dtype=torch.float64, device=fsd.device)
        self._c(A.lib().rt_set_force_support(self._h, _dp(fsd), _dp(f)))
        self.ctx.sync()
        return f.cpu().numpy()

    def displacementProject(self, u):
        """displacementProject (optimization/projection.cpp:374-392): u minus its rigid-mode part
        (no-support modes)."""
        ud = self._dev(u)
        self._c(A.lib().rt_displacement_project(self._h, _dp(ud)))
        self.ctx.sync()
        return ud.cpu().numpy()

    # design state files (the reference writes OpenVDB grids, grid/Grid.cpp:727-839, and raw
    # vectors, utils/binaryIO.h) -------------------------------------------------------------
    def write_state(self, path, fields=("rho", "u", "f"), **meta):
        """Writes the level-0 fields as .npy files into directory ``path`` with a manifest.json
        (grid sizes, field files, the activity checksum and ``meta``: e.g. the iteration and the
        worst-case eigenvalue).  Returns the manifest."""
        import hashlib
        import json
        import os

        os.makedirs(path, exist_ok=True)
        g0 = self[0]
        get = {"rho": g0.getRho, "u": g0.getDisplacement, "f": g0.getForce, "sens": g0.getSens}
        files = {}
        for name in fields:
            np.save(os.path.join(path, f"{name}.npy"), get[name]())
            files[name] = f"{name}.npy"
        man = {"format": "robtop_b200 state 1", "dims": [g0.nx, g0.ny, g0.nz], "n_levels": self.n_grid(),
               "mode": int(self.params.mode), "eact_sha1": hashlib.sha1(g0.getEact().tobytes()).hexdigest(),
               "fields": files, "meta": meta}
        with open(os.path.join(path, "manifest.json"), "w") as fp:
            json.dump(man, fp, indent=1)
        return man

    def read_state(self, path):
        """Loads a state written by write_state into this hierarchy (same grid); returns the manifest."""
        import hashlib
        import json
        import os

        with open(os.path.join(path, "manifest.json")) as fp:
            man = json.load(fp)
        g0 = self[0]
        if man.get("format") != "robtop_b200 state 1" or man["dims"] != [g0.nx, g0.ny, g0.nz]:
            raise ValueError(f"{path}: not a state of a {g0.nx}x{g0.ny}x{g0.nz} grid")
        if man["eact_sha1"] != hashlib.sha1(g0.getEact().tobytes()).hexdigest():
            raise ValueError(f"{path}: written for a different solid")
        put = {"rho": g0.setRho, "u": g0.setDisplacement, "f": g0.setForce, "sens": g0.setSens}
        for name, fn in man["fields"].items():
            put[name](np.load(os.path.join(path, fn)))
        return man

    def workspace(self):
        """A solve workspace sharing this hierarchy's operator (rt_hier_workspace_create)."""
        ws = HierarchyGrid(self.ctx, self.params)
        self._c(A.lib().rt_hier_workspace_create(self._h, C.byref(ws._h)))
        ws._init_levels()
        ws._parent = self  # destroyed before the parent
        self._children.append(ws)
        return ws

    def close(self):
        for ws in getattr(self, "_children", []):
            ws.close()
        self._children = []
        if self._h:
            A.lib().rt_hier_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def voxelize_mesh(ctx, pcoords, facevertices, prefer_reso):
    """voxelize_mesh (voxelizer/voxelize_main.cpp:344-402) on the device: returns the solid
    bits (most significant bit first in each word, bit x + y R + z R^2), R and the cube
    ``[[min xyz], [max xyz]]``."""
    v = np.ascontiguousarray(pcoords, np.float32).reshape(-1)
    f = np.ascontiguousarray(facevertices, np.int32).reshape(-1)
    R = A.lib().rt_voxel_resolution(int(prefer_reso))
    if R == 0:
        raise ValueError("prefer_reso must be in [1, 1023]")
    bits = np.zeros((R ** 3 + 31) // 32, np.uint32)
    reso = np.zeros(3, np.int32)
    box = np.zeros(6, np.float32)
    check(A.lib().rt_voxelize_mesh(ctx.handle, _p(v), v.size // 3, _p(f), f.size // 3, int(prefer_reso), _p(bits),
                                   bits.size, _p(reso), _p(box)), ctx.handle)
    return bits, int(reso[0]), box.reshape(2, 3)


def pcg_batch(grids, tol=1e-6, maxit=500):
    """rt_pcg_batch: u <- K^-1 f on every hierarchy / workspace in one graph launch."""
    hs = (C.c_void_p * len(grids))(*[g.handle.value for g in grids])
    infos = (A.SolveInfo * len(grids))()
    st = A.lib().rt_pcg_batch(hs, len(grids), tol, maxit, infos)
    if st not in (A.RT_OK, A.RT_ENOCONV):
        check(st, grids[0].ctx.handle)
    return list(infos)
