"""Python mirror of robtop's optimization module (optimization/optimization.h:28-82).

Module-level state stands in for the reference's globals ``grids`` and
``params`` (optimization/optimization.cpp:8-12); every numeric step runs in
``librtb200.so`` through :mod:`robtop_b200.grid`.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi as A
from .grid import Context, HierarchyGrid, default_params


@dataclass
class Parameter:
    """optimization/optimization.h:11-22"""
    damp_ratio: float = 0.5
    design_step: float = 0.03
    power_penalty: float = 3.0
    volume_ratio: float = 0.4
    volume_decrease: float = 0.0
    filter_radius: int = 2
    min_rho: float = 1e-3
    gridreso: int = 128
    youngs_modulu: float = 1e6
    poisson_ratio: float = 0.4
    shell_width: float = 3.0  # elements within this many element lengths of the mesh surface stay solid


params = Parameter()
_state = {"ctx": None, "grids": None, "mode": A.MODE_WSFF, "fixed": None, "load": None, "field": None,
          "pm_seed": 1, "records": []}


def _ctx():
    if _state["ctx"] is None:
        _state["ctx"] = Context(0)
    return _state["ctx"]


def getGrids() -> HierarchyGrid:
    return _state["grids"]


def setParameters(volRatio, volDecrease, designStep, filterRadi, dampRatio, powerPenal, min_density, gridreso,
                  youngs_modulu, poisson_ratio, shell_width=0.0, logdensity=False, logcompliance=False):
    """optimization/optimization.cpp:32-50"""
    params.volume_ratio = volRatio
    params.volume_decrease = volDecrease
    params.design_step = designStep
    params.filter_radius = int(filterRadi)
    params.damp_ratio = dampRatio
    params.power_penalty = powerPenal
    params.min_rho = min_density
    params.gridreso = gridreso
    params.youngs_modulu = youngs_modulu
    params.poisson_ratio = poisson_ratio
    params.shell_width = shell_width


def setWorkMode(modestr):
    """optimization/optimization.cpp:65-83 (raises instead of exit(-1))."""
    modes = {"nscf": A.MODE_NSCF, "nsff": A.MODE_NSFF, "wscf": A.MODE_WSCF, "wsff": A.MODE_WSFF}
    if modestr not in modes:
        raise ValueError(f"unsupported mode {modestr}")
    _state["mode"] = modes[modestr]
    if _state["grids"] is not None:
        _state["grids"].setMode(modes[modestr])


def setBoundaryCondition(fixarea, loadarea, forcefield):
    """optimization/optimization.cpp:680-685; predicates take a position (x, y, z)."""
    _state["fixed"], _state["load"], _state["field"] = fixarea, loadarea, forcefield


def _rt_params(**kw):
    return default_params(power_penalty=params.power_penalty, min_rho=params.min_rho,
                          volume_ratio=params.volume_ratio, design_step=params.design_step,
                          damp_ratio=params.damp_ratio, filter_radius=float(params.filter_radius),
                          youngs_modulus=params.youngs_modulu, poisson_ratio=params.poisson_ratio,
                          mode=_state["mode"], skip_layer1=1, **kw)


def _word_reverse(words):
    """Most-significant-bit-first words -> least-significant-bit-first (wordReverse_g)."""
    b = np.ascontiguousarray(words, np.uint32).view(np.uint8).reshape(-1, 4)
    rev = np.unpackbits(b, axis=1, bitorder="little")[:, ::-1]  # bit 31 .. 0 of each word
    return np.packbits(rev, axis=1, bitorder="little").reshape(-1).view(np.uint32).copy()


def _predicate(fn, pos):
    """Applies a region predicate: vectorised (``contains``) or one position at a time."""
    if fn is None:
        return np.zeros(len(pos), bool)
    if hasattr(fn, "contains"):
        return np.asarray(fn.contains(pos), bool)
    return np.array([bool(fn(p)) for p in pos], bool)


def buildGrids(a, b, **solver):
    """Builds the hierarchy and applies the boundary predicates to the level-0 surface nodes
    (Grid::computeProjectionMatrix, grid/Grid.cpp:1291-1403).

    ``buildGrids(coords, trifaces)`` (optimization/optimization.cpp:14-19): the closed triangle
    mesh is voxelised on the device at ``params.gridreso`` and node positions are in the mesh
    frame (cube corner + node index x element length).  ``buildGrids(solid_bit, reso)``: a
    cubic bit grid (genFromMesh(solid_bit, out_reso), grid/Grid.cpp:455), least significant bit
    first; node positions are the node indices."""
    G = HierarchyGrid(_ctx(), _rt_params(**solver))
    if np.isscalar(b):
        reso = int(b)
        G.genFromMesh(a, [reso, reso, reso])
        origin, h = np.zeros(3), np.ones(3)
    else:
        from .grid import voxelize_mesh

        bits, reso, box = voxelize_mesh(_ctx(), a, b, params.gridreso)
        G.genFromMesh(_word_reverse(bits), [reso, reso, reso])
        origin = box[0].astype(np.float64)
        h = (box[1].astype(np.float64) - origin) / reso
        _state["box"] = box
        _state["mesh"] = (np.asarray(a, np.float32).reshape(-1, 3), np.asarray(b, np.int32).reshape(-1, 3))
    g0 = G[0]
    surf = G.surface_nodes().astype(bool) & g0.getVact().astype(bool)
    nv = g0.nv
    vx, vy = g0.nx + 1, g0.ny + 1
    ids = np.flatnonzero(surf)
    pos = origin + np.stack([ids % vx, (ids // vx) % vy, ids // (vx * vy)], 1).astype(np.float64) * h
    fixed = _predicate(_state["fixed"], pos)
    loadm = _predicate(_state["load"], pos)
    loadm &= ~fixed
    vfix = np.zeros(nv, np.uint8)
    vfix[ids[fixed]] = 1
    G.set_support(vfix)
    load_ids = ids[loadm]
    if np.isscalar(b):
        normals = np.tile([0.0, 0.0, 1.0], (load_ids.size, 1))
    else:
        # Grid::outwardNormal (closest surface point), and the shell elements of
        # HierarchyGrid::setSolidShellElement (grid/Grid.cpp:67-137, 1404-1423)
        from .boundary import outward_normals, shell_elements

        mv, mf = _state["mesh"]
        normals = outward_normals(pos[loadm], mv, mf) if load_ids.size else np.zeros((0, 3))
        eact = g0.getEact().reshape(g0.nz, g0.ny, g0.nx)
        if params.shell_width > 0:
            G.set_shell(shell_elements(eact, origin, h, mv, mf, params.shell_width).ravel())
    G.set_load_nodes(load_ids, normals)
    _state["grids"] = G
    _state["fixed_ids"] = ids[fixed]
    _state["load_ids"] = load_ids
    _state["load_pos"] = pos[loadm]
    return G


def uploadTemplateMatrix():
    G = getGrids()
    p = G.params
    p.youngs_modulus, p.poisson_ratio, p.power_penalty = params.youngs_modulu, params.poisson_ratio, \
        params.power_penalty
    G.set_params(p)


def initDensities(rho):
    getGrids()[0].init_rho(rho)


def update_stencil():
    getGrids().update_stencil()


def solveFEM(tol=1e-4):
    """optimization/optimization.cpp:85-91 on the preloaded force field."""
    G = getGrids()
    nv = G[0].nv
    f = np.zeros(3 * nv)
    field = _state["field"]
    if field is not None and hasattr(field, "force"):  # a parsed configuration's summed fields
        vals = field.force(_state["load_pos"]) if len(_state["load_pos"]) else np.zeros((0, 3))
    else:
        vals = [field(p) if field else (0.0, 0.0, 0.0) for p in _state["load_pos"]]
    for i, v in zip(_state["load_ids"], vals):
        f[i], f[nv + i], f[2 * nv + i] = v
    G[0].setForce(f)
    rel = 1.0
    it = 0
    while rel > tol:
        rel = G.v_cycle()
        it += 1
        if it > 1000 or not np.isfinite(rel):
            raise RuntimeError("solveFEM did not converge")
    return rel


def modifiedPM():
    """optimization/optimization.cpp:123-261 (on the device)."""
    lam, _ = getGrids().worst_case(A.WORST_MODPM, 500, 0.0, seed=_state["pm_seed"])
    _state["pm_seed"] += 1
    return lam


def worstCaseLanczos(k=16, inner_tol=1e-6, seed=0):
    lam, _ = getGrids().worst_case(A.WORST_LANCZOS, k, inner_tol, seed=seed)
    return lam


def computeSensitivity():
    A.check(A.lib().rt_sensitivity(getGrids().handle, 1), _ctx().handle)


def updateDensities(Vgoal):
    lam = C.c_float()
    trials = C.c_int()
    A.check(A.lib().rt_oc_update(getGrids().handle, float(Vgoal), C.byref(lam), C.byref(trials)), _ctx().handle)
    return lam.value


def setOutpurDir(dirname):
    """optimization/optimization.cpp (setOutpurDir): where optimization() writes its checkpoints."""
    _state["outdir"] = dirname


def writeDensity(path):
    """The design state (densities, displacement, force) as .npy files with a manifest
    (HierarchyGrid::writeDensity, grid/Grid.cpp:727-764, writes an OpenVDB grid instead)."""
    return getGrids().write_state(path, iteration=_state.get("iteration", 0), records=_state["records"])


def readDensity(path):
    """Loads a state written by writeDensity (HierarchyGrid::readDensity, grid/Grid.cpp:809-839)."""
    man = getGrids().read_state(path)
    _state["records"] = list(man["meta"].get("records", []))
    _state["iteration"] = int(man["meta"].get("iteration", 0))
    return man


class ConvergeCriteria:
    """snippet::converge_criteria (utils/snippet.h:156-213): the stop test of optimization().

    Each update records the objective c_k and the constraint values g_k.  The objective change
    fch = |c_k + c_{k-1} - c_{k-2} - c_{k-3}| / (c_{k-2} + c_{k-3}) (not a number while fewer
    than four values exist) must be below ``stop_thres`` and each constraint's change, formed
    the same way, must not exceed 1e-3.  A passing update raises a counter, a failing one lowers
    it (not below 0); update returns True once the counter exceeds ``max_counter``.

    ``integer_abs`` reproduces the header as g++ compiles it: its unqualified abs() of the
    change resolves to the C library's int abs(int), so the numerator is truncated to an integer
    first and every change below 1 reads as 0.  The default is the floating-point change (the
    header under MSVC, and the test as it is written)."""

    def __init__(self, n_constrain, max_counter, stop_thres, integer_abs=False):
        self.n = int(n_constrain)
        self.max_counter = int(max_counter)
        self.thres = float(stop_thres)
        self.integer_abs = bool(integer_abs)
        self.values, self.constraints = [], []
        self.counter = 0

    def _change(self, h):
        if len(h) < 4:
            return float("nan")
        a, b, c, d = h[-1], h[-2], h[-3], h[-4]
        num, den = np.float64(a + b - c - d), np.float64(c + d)
        if self.integer_abs and np.isfinite(num):
            num = np.trunc(num)
        with np.errstate(divide="ignore", invalid="ignore"):
            return float(np.abs(num) / den)

    def update(self, value, constraints=()):
        self.values.append(float(value))
        self.constraints.append([float(g) for g in constraints][: self.n])
        converged = self._change(self.values) < self.thres
        for i in range(self.n):
            if self._change([g[i] for g in self.constraints]) > 1e-3:
                converged = False
                break
        self.counter = self.counter + 1 if converged else max(self.counter - 1, 0)
        return self.counter > self.max_counter


def optimization(max_iter=100, worst=modifiedPM, checkpoint_every=0, resume=None):
    """optimization/optimization.cpp:583-673; returns the worst-case compliance record.

    Per iteration: the volume goal shrinks by volume_decrease (the constraint value Vc recorded
    for the stop test is taken before the goal is clamped to volume_ratio), the stencils are
    updated, the worst-case compliance is found, and the loop ends when
    converge_criteria(1, 2, 5e-3) reports convergence with the goal at the volume ratio;
    otherwise sensitivity, filter and OC update follow.  The volume goals are kept in
    ``_state["volumes"]``.  With ``checkpoint_every`` = n > 0 the state is written every n
    iterations into <output dir>/iter_<k> (setOutpurDir); ``resume`` = such a directory
    continues from it (the stop test replays the recorded values)."""
    import os

    rec, vols, start = [], [], 1
    if resume:
        readDensity(resume)
        rec, start = list(_state["records"]), _state["iteration"] + 1
    else:
        initDensities(params.volume_ratio)
    stop = ConvergeCriteria(1, 2, 5e-3)
    Vgoal = params.volume_ratio
    for c in rec:  # a resumed run: the stop test and the goals of the recorded iterations
        Vgoal *= 1 - params.volume_decrease
        stop.update(c, [Vgoal - params.volume_ratio])
        Vgoal = max(Vgoal, params.volume_ratio)
        vols.append(Vgoal)
    for itn in range(start, max_iter + 1):
        _state["iteration"] = itn
        Vgoal *= 1 - params.volume_decrease
        Vc = Vgoal - params.volume_ratio
        Vgoal = max(Vgoal, params.volume_ratio)
        update_stencil()
        c = worst()
        rec.append(c)
        vols.append(Vgoal)
        _state["records"], _state["volumes"] = rec, vols
        if stop.update(c, [Vc]) and Vgoal <= params.volume_ratio + 1e-3:
            break
        computeSensitivity()
        updateDensities(Vgoal)
        if checkpoint_every and itn % checkpoint_every == 0:
            writeDensity(os.path.join(_state.get("outdir", "."), f"iter_{itn}"))
    _state["records"], _state["volumes"] = rec, vols
    return rec


def run_config(jsonfile, meshfile=None, workmode="wsff", max_iter=100, worst=modifiedPM, **flags):
    """The robtop.cpp flow driven by a benchmark configuration (config_parser_t::parse,
    config_parser.cpp:485-498, then robtop.cpp:27-46): parse the regions and force fields,
    read the mesh (the configuration's ``model`` unless ``meshfile`` is given), set the
    parameters (``flags`` as setParameters' keywords), build the grids from the mesh and run
    the optimisation.  Returns the compliance record."""
    from .boundary import parse_config, read_mesh

    cfg = parse_config(jsonfile)
    path = meshfile or cfg.model_path()
    if not path:
        raise ValueError("no mesh: the configuration names no model and no meshfile was given")
    v, f = read_mesh(path)
    kw = dict(volRatio=0.3, volDecrease=0.02, designStep=0.03, filterRadi=2, dampRatio=0.5, powerPenal=3.0,
              min_density=1e-3, gridreso=200, youngs_modulu=1e6, poisson_ratio=0.4,
              shell_width=3.0)  # the reference's flag defaults
    kw.update(flags)
    setParameters(**kw)
    setWorkMode(workmode)
    setBoundaryCondition(cfg.fixed_area, cfg.load_area, cfg)
    buildGrids(v, f)
    uploadTemplateMatrix()
    return optimization(max_iter=max_iter, worst=worst)
