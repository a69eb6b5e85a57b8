"""Host-side mirror of the reference's public API (lagrangian/src/PlasticityFEM.jl:35-47).

Names and argument meanings follow the Julia package: ``box_mesh``, ``on_face``,
``select_nodes``, ``J2Material``, ``Model``, ``fix``/``prescribe``/``load``
(Julia ``fix!``/``prescribe!``/``load!``), ``solve`` (``solve!``), ``reset``,
``nodal_displacements``, ``gauss_stress``, ``gauss_kirchhoff``,
``equivalent_plastic_strain``, ``assemble`` (``assemble!``).  Every numerical
call goes through the C ABI of ``libpfem_b200.so``; this module only moves
host arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from . import _lib as L
from ._lib import check, ptr


# ------------------------------------------------------------------ mesh (Mesh.jl)
@dataclass
class Mesh:
    """Mesh (Mesh.jl:17-22): nodes 3 x nn (float64), elements 8 x ne (1-based int64)."""
    nodes: np.ndarray
    elements: np.ndarray

    @property
    def nnodes(self) -> int:
        return self.nodes.shape[1]

    @property
    def nelem(self) -> int:
        return self.elements.shape[1]


def box_mesh(lx, ly, lz, nx: int, ny: int, nz: int) -> Mesh:
    """box_mesh (Mesh.jl:30-59): lexicographic nodes (x fastest), VTK Hex8 order."""
    npx, npy = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    nodes = np.stack([float(lx) * i.ravel() / nx, float(ly) * j.ravel() / ny,
                      float(lz) * k.ravel() / nz]).astype(np.float64)
    ke, je, ie = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ie, je, ke = ie.ravel(), je.ravel(), ke.ravel()

    def nid(i, j, k):
        return (k * npy + j) * npx + i + 1

    el = np.stack([nid(ie, je, ke), nid(ie + 1, je, ke), nid(ie + 1, je + 1, ke),
                   nid(ie, je + 1, ke), nid(ie, je, ke + 1), nid(ie + 1, je, ke + 1),
                   nid(ie + 1, je + 1, ke + 1), nid(ie, je + 1, ke + 1)]).astype(np.int64)
    return Mesh(nodes, el)


def select_nodes(mesh: Mesh, pred) -> np.ndarray:
    """select_nodes (Mesh.jl:66-74): 1-based ids where pred(x, y, z) holds."""
    x, y, z = mesh.nodes
    mask = np.asarray(pred(x, y, z), dtype=bool)
    return np.nonzero(mask)[0].astype(np.int64) + 1


def on_face(mesh: Mesh, face: str) -> np.ndarray:
    """on_face (Mesh.jl:82-104), tolerance 1e-8 * max(L, 1)."""
    face = face.lstrip(":")
    x, y, z = mesh.nodes
    lo = mesh.nodes.min(axis=1)
    hi = mesh.nodes.max(axis=1)
    Lmax = float(np.max(hi - lo))
    tol = 1e-8 * max(Lmax, 1.0)
    ax = {"x": 0, "y": 1, "z": 2}[face[0]]
    v = lo[ax] if face.endswith("min") else hi[ax]
    if not (face.endswith("min") or face.endswith("max")):
        raise ValueError(f"unknown face {face}")
    return np.nonzero(np.abs(mesh.nodes[ax] - v) <= tol)[0].astype(np.int64) + 1


def dof(node, comp):
    """dof (Mesh.jl:111): 3(node-1) + comp, both 1-based."""
    return 3 * (np.asarray(node) - 1) + np.asarray(comp)


# ------------------------------------------------------------------ material
@dataclass
class J2Material:
    """J2Material (Materials.jl:68-108): isotropic hardening
    sigma_y(a) = sigy0 + (sigsat - sigy0)(1 - exp(-delta a)) + Hiso a (yield_stress,
    :117-118; linear when delta = 0 or sigsat = sigy0) and linear kinematic hardening Hkin."""
    E: float
    nu: float
    sigy0: float
    Hiso: float = 0.0
    Hkin: float = 0.0
    sigsat: float | None = None   # keyword default: sigy0
    delta: float = 0.0

    def __post_init__(self):
        # ArgumentError guards, Materials.jl:90-103
        if not self.E > 0:
            raise ValueError(f"E must be positive (got {self.E})")
        if not (-1 < self.nu < 0.5):
            raise ValueError(f"nu must satisfy -1 < nu < 0.5 (got {self.nu})")
        if not self.sigy0 > 0:
            raise ValueError(f"sigy0 must be positive (got {self.sigy0})")
        if self.Hiso < 0 or self.Hkin < 0:
            raise ValueError("hardening moduli must be >= 0")
        if self.sigsat is None:
            self.sigsat = self.sigy0
        if not self.sigsat >= self.sigy0:
            raise ValueError(f"sigsat must be >= sigy0 (got sigsat={self.sigsat}, sigy0={self.sigy0})")
        if not self.delta >= 0:
            raise ValueError(f"delta must be >= 0 (got {self.delta})")
        if self.delta > 0 and self.sigsat > self.sigy0 and self.Hkin > 0:
            raise ValueError("saturation hardening (sigsat>sigy0, delta>0) with kinematic hardening "
                             "(Hkin>0) is not supported; use one or the other")

    def yield_stress(self, a):
        """yield_stress (Materials.jl:117-118)."""
        return self.sigy0 + (self.sigsat - self.sigy0) * (1 - np.exp(-self.delta * a)) + self.Hiso * a

    @property
    def G(self):
        return self.E / (2 * (1 + self.nu))

    @property
    def lam(self):
        return self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))

    def _c(self) -> L.Material:
        return L.Material(self.E, self.nu, self.sigy0, self.Hiso, self.Hkin, self.sigsat, self.delta)


@dataclass
class SolveResult:
    """SolveResult (Solver.jl:61-66) plus device timings."""
    converged: bool
    iters: list
    residuals: list
    cg_iters: list
    stats: dict = field(default_factory=dict)


_KINDS = {"small": L.PFEM_HEX8_SMALL, "finite": L.PFEM_HEX8_FINITE, "finite_fbar": L.PFEM_HEX8_FINITE_FBAR}
_PREC = {"fp64": L.PFEM_FP64, "mixed": L.PFEM_MIXED}
_PRED = {"previous": L.PFEM_PRED_PREVIOUS, "extrapolate": L.PFEM_PRED_EXTRAPOLATE,
         "learned": L.PFEM_PRED_LEARNED}
_KRY = {"cg": L.PFEM_KRYLOV_CG, "bicgstab": L.PFEM_KRYLOV_BICGSTAB}


class Model:
    """Model(mesh, material; element=:finite_fbar) (Model.jl:63-75), on one GPU.

    ``sigy0_e`` optionally gives a per-element initial yield stress.
    """

    def __init__(self, mesh: Mesh, material: J2Material, element: str = "finite_fbar",
                 sigy0_e=None, device: int = 0):
        element = element.lstrip(":")
        if element not in _KINDS:
            raise ValueError(f"unknown element kind {element} (use small, finite, finite_fbar)")
        self.mesh = mesh
        self.material = material
        self.element = element
        self.nn, self.ne = mesh.nnodes, mesh.nelem
        self.ndof, self.ngp = 3 * self.nn, 8 * self.ne
        nodes = np.ascontiguousarray(mesh.nodes.T, dtype=np.float64)        # (nn,3) = 3 x nn col-major
        els = np.ascontiguousarray(mesh.elements.T, dtype=np.int64)          # (ne,8) = 8 x ne col-major
        sy = None if sigy0_e is None else np.ascontiguousarray(sigy0_e, dtype=np.float64)
        self._ctx = C.c_void_p()
        m = material._c()
        rc = L.lib().pfem_create(C.byref(self._ctx), ptr(nodes), self.nn, ptr(els, L._i64), self.ne,
                                 _KINDS[element], C.byref(m), ptr(sy), device)
        check(rc, None)
        self.dir_dofs, self.dir_vals, self.dir_ramp = [], [], []
        self.neu_dofs, self.neu_vals = [], []
        self._bcs_dirty = True

    _BC_FIELDS = frozenset(("dir_dofs", "dir_vals", "dir_ramp", "neu_dofs", "neu_vals"))

    def __setattr__(self, name, value):
        # Replacing a boundary-condition list (as Workload.apply does) must
        # reach the device before the next solve, like the fix!/prescribe!/load!
        # builders do (Model.jl:102-145; frozen by _freeze_bcs, Solver.jl:192-218).
        object.__setattr__(self, name, value)
        if name in Model._BC_FIELDS:
            object.__setattr__(self, "_bcs_dirty", True)

    def __del__(self):
        ctx = getattr(self, "_ctx", None)
        if ctx is not None and ctx.value:
            try:
                L.lib().pfem_destroy(ctx)
            except Exception:
                pass
            self._ctx = None

    # --- BC builders (Model.jl:102-145) ---
    @staticmethod
    def _comps(comp):
        comp = comp.lstrip(":")
        return {"x": (1,), "y": (2,), "z": (3,), "all": (1, 2, 3)}[comp]

    def _dofs(self, nodes, comp):
        """1-based dofs of `nodes` x `comp`, node-major (the order of the
        reference builders' nested loops)."""
        nodes = np.atleast_1d(np.asarray(nodes, np.int64))
        comps = np.asarray(self._comps(comp), np.int64)
        return (3 * (nodes[:, None] - 1) + comps[None, :]).reshape(-1)

    def _extend(self, **arrays):
        # the lists may be numpy arrays (Workload.apply assigns arrays)
        for name, add in arrays.items():
            cur = getattr(self, name)
            setattr(self, name, np.concatenate([np.asarray(cur, add.dtype), add]))

    def fix(self, nodes, comp="all"):
        d = self._dofs(nodes, comp)
        self._extend(dir_dofs=d, dir_vals=np.zeros(len(d)), dir_ramp=np.zeros(len(d), np.uint8))
        return self

    def prescribe(self, nodes, comp, value, ramp=True):
        d = self._dofs(nodes, comp)
        self._extend(dir_dofs=d, dir_vals=np.full(len(d), float(value)),
                     dir_ramp=np.full(len(d), 1 if ramp else 0, np.uint8))
        return self

    def load(self, nodes, comp, value, distribute=False):
        nodes = np.atleast_1d(nodes)
        per = float(value) / len(nodes) if distribute else float(value)
        d = self._dofs(nodes, comp)
        self._extend(neu_dofs=d, neu_vals=np.full(len(d), per))
        return self

    def _push_bcs(self):
        if not self._bcs_dirty:
            return
        dd = np.asarray(self.dir_dofs, np.int64); dv = np.asarray(self.dir_vals, np.float64)
        dr = np.asarray(self.dir_ramp, np.uint8)
        nd = np.asarray(self.neu_dofs, np.int64); nv = np.asarray(self.neu_vals, np.float64)
        rc = L.lib().pfem_set_bcs(self._ctx, ptr(dd, L._i64), ptr(dv), ptr(dr, L._u8), len(dd),
                                  ptr(nd, L._i64), ptr(nv), len(nd))
        check(rc, self._ctx)
        self._bcs_dirty = False

    # --- structure ---
    def pattern(self):
        """1-based CSC colptr/rowval (int64) of SparsityPattern.K (Assembly.jl:99-148)."""
        nnz = C.c_int64()
        check(L.lib().pfem_pattern(self._ctx, C.byref(nnz), None, None), self._ctx)
        colptr = np.zeros(self.ndof + 1, np.int64)
        rowval = np.zeros(nnz.value, np.int64)
        check(L.lib().pfem_pattern(self._ctx, C.byref(nnz), ptr(colptr, L._i64), ptr(rowval, L._i64)),
              self._ctx)
        return colptr, rowval

    def colors(self):
        nc = C.c_int32()
        col = np.zeros(self.ne, np.int64)
        check(L.lib().pfem_colors(self._ctx, C.byref(nc), ptr(col, L._i64)), self._ctx)
        return nc.value, col

    # --- hot path ---
    def assemble(self, U, commit=False, precision="fp64", want_K=True):
        """assemble! (Assembly.jl:238-257) -> (K scipy.csr or None, R, tau (ngp,6), flags)."""
        U = np.ascontiguousarray(U, np.float64)
        R = np.zeros(self.ndof)
        tau = np.zeros((self.ngp, 6))
        fl = np.zeros(self.ngp, np.uint8)
        K = None
        if want_K and not commit:
            colptr, rowval = self.pattern()
            kv = np.zeros(len(rowval))
            rc = L.lib().pfem_assemble(self._ctx, ptr(U), int(commit), _PREC[precision], ptr(R), ptr(kv),
                                       ptr(tau), ptr(fl, L._u8))
            check(rc, self._ctx)
            K = sp.csr_matrix((kv, rowval - 1, colptr - 1), shape=(self.ndof, self.ndof))
        else:
            rc = L.lib().pfem_assemble(self._ctx, ptr(U), int(commit), _PREC[precision], ptr(R), None,
                                       ptr(tau), ptr(fl, L._u8))
            check(rc, self._ctx)
        return K, R, tau, fl

    def _opts(self, nsteps=10, tol=1e-8, maxiter=25, precision="fp64", linsolve="cg", lin_rtol=None,
              predictor="previous", amg_rebuild=None, cheb_degree=2, cg_itmax=200, eta_min=None,
              line_search=False, verbose=False, predictor_smooth=None, eta_max=None, max_cuts=0,
              eta_first=None, amg_stale_ratio=None, ew_need=None):
        o = L.SolveOpts()
        L.lib().pfem_default_opts(C.byref(o))
        o.nsteps, o.maxiter, o.tol = nsteps, maxiter, tol
        o.precision = _PREC[precision]
        o.krylov = _KRY[linsolve]
        o.lin_rtol = -1.0 if lin_rtol is None else float(lin_rtol)
        if eta_min is not None:
            o.eta_min = eta_min
        elif precision == "mixed":
            o.eta_min = 1e-6   # FP32 inner solves cannot go much below this
        o.predictor = _PRED[predictor]
        if amg_rebuild is not None:
            o.amg_rebuild = 2 if amg_rebuild == "adaptive" else int(bool(amg_rebuild))
        if amg_stale_ratio is not None:
            o.amg_stale_ratio = float(amg_stale_ratio)
        if ew_need is not None:
            o.ew_need = int(bool(ew_need))
        o.cheb_degree = cheb_degree
        o.krylov_itmax = cg_itmax
        o.verbose = int(bool(verbose))
        o.line_search = int(bool(line_search))
        if predictor_smooth is not None:
            o.predictor_smooth = int(predictor_smooth)
        if eta_max is not None:
            o.eta_max = float(eta_max)
        o.max_cuts = int(max_cuts)
        if eta_first is not None:
            o.eta_first = float(eta_first)
        return o

    def solve(self, nsteps=10, tol=1e-8, maxiter=25, **kw) -> SolveResult:
        """solve! (Solver.jl:419-475) on the GPU."""
        self._push_bcs()
        o = self._opts(nsteps=nsteps, tol=tol, maxiter=maxiter, **kw)
        res = L.SolveResultC()
        its = np.zeros(nsteps, np.int32)
        hist = np.zeros((nsteps, maxiter))
        kh = np.zeros((nsteps, maxiter), np.int32)
        rc = L.lib().pfem_solve(self._ctx, C.byref(o), C.byref(res), ptr(its, L._i32), ptr(hist),
                                ptr(kh, L._i32))
        if rc not in (L.PFEM_OK, L.PFEM_ERR_NOT_CONVERGED):
            check(rc, self._ctx)
        n = max(res.steps_done + (0 if res.converged else 1), 0)
        iters = [int(i) for i in its[:n]]
        residuals = [list(hist[s, :iters[s]]) for s in range(n)]
        cg = [list(map(int, kh[s, :max(iters[s] - 1, 0)])) for s in range(n)]
        stats = {k: getattr(res, k) for k, _ in L.SolveResultC._fields_}
        return SolveResult(bool(res.converged), iters, residuals, cg, stats)

    def newton(self, lam, **kw):
        """newton! (Solver.jl:317-389) for one load step + commit."""
        self._push_bcs()
        o = self._opts(**kw)
        it = C.c_int32()
        hist = np.zeros(o.maxiter)
        kh = np.zeros(o.maxiter, np.int32)
        rc = L.lib().pfem_newton(self._ctx, float(lam), C.byref(o), C.byref(it), ptr(hist), ptr(kh, L._i32))
        check(rc, self._ctx)
        return list(hist[:it.value]), list(kh[:max(it.value - 1, 0)])

    def predict(self, lam, predictor="learned", **kw):
        """Newton predictor for the load step to `lam` alone (no reference counterpart):
        leaves the chosen guess as the current U and returns
        (U, |R| extrapolated, |R| learned or None, learned guess kept)."""
        self._push_bcs()
        o = self._opts(predictor=predictor, **kw)
        U = np.zeros(self.ndof)
        rex, rml, used = C.c_double(), C.c_double(), C.c_int32()
        check(L.lib().pfem_predict(self._ctx, float(lam), C.byref(o), ptr(U), C.byref(rex), C.byref(rml),
                                   C.byref(used)), self._ctx)
        return U, rex.value, (rml.value if rml.value >= 0 else None), bool(used.value)

    def residual(self, lam, precision="fp64"):
        """Assemble + impose at the current U (one newton! iteration's residual);
        leaves the imposed tangent resident.  Returns (||R||, R)."""
        self._push_bcs()
        R = np.zeros(self.ndof)
        rn = C.c_double()
        check(L.lib().pfem_residual(self._ctx, float(lam), _PREC[precision], C.byref(rn), ptr(R)), self._ctx)
        return rn.value, R

    def linear_solve(self, b, rtol, rebuild=True, **kw):
        o = self._opts(**kw)
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.ndof)
        n = C.c_int32()
        rc = L.lib().pfem_linear_solve(self._ctx, ptr(b), ptr(x), float(rtol), int(rebuild), C.byref(o),
                                       C.byref(n))
        check(rc, self._ctx)
        return x, n.value

    def amg_apply(self, r):
        """One cycle of the resident AMG hierarchy (V on level 0, W below): z = M^-1 r."""
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros(self.ndof)
        check(L.lib().pfem_amg_apply(self._ctx, ptr(r), ptr(z)), self._ctx)
        return z

    def amg_dense(self, level, what):
        """Dense copy of an AMG operator (what=0), prolongator (what=1) or, on the
        coarsest level, the dense inverse the cycle applies (what=2)."""
        dims = np.zeros(2, np.int64)
        check(L.lib().pfem_amg_dense(self._ctx, level, what, None, ptr(dims, L._i64)), self._ctx)
        out = np.zeros((int(dims[0]), int(dims[1])))
        check(L.lib().pfem_amg_dense(self._ctx, level, what, ptr(out), ptr(dims, L._i64)), self._ctx)
        return out

    def reset(self):
        check(L.lib().pfem_reset(self._ctx), self._ctx)
        return self

    def set_state(self, cpi=None, alpha=None, epsp=None):
        """Overwrite the committed per-GP state (arrays shaped (ngp, 6) / (ngp,))."""
        c = None if cpi is None else np.ascontiguousarray(cpi, np.float64)
        a = None if alpha is None else np.ascontiguousarray(alpha, np.float64)
        e = None if epsp is None else np.ascontiguousarray(epsp, np.float64)
        check(L.lib().pfem_set_state(self._ctx, ptr(c), ptr(a), ptr(e)), self._ctx)

    def back_stress(self):
        """Committed back stress (GaussState.beta, Mesh.jl:124-130), shape (ngp, 6);
        the rotation-neutralised (reference-configuration) back stress for the
        finite kinds, zeros when Hkin = 0."""
        b = np.zeros((self.ngp, 6))
        check(L.lib().pfem_get_back_stress(self._ctx, ptr(b)), self._ctx)
        return b

    def set_back_stress(self, beta):
        b = np.ascontiguousarray(beta, np.float64)
        check(L.lib().pfem_set_back_stress(self._ctx, ptr(b)), self._ctx)

    def set_displacement(self, U):
        U = np.ascontiguousarray(U, np.float64)
        check(L.lib().pfem_set_displacement(self._ctx, ptr(U)), self._ctx)

    def state(self):
        U = np.zeros(self.ndof)
        tau = np.zeros((self.ngp, 6)); cpi = np.zeros((self.ngp, 6)); ep = np.zeros((self.ngp, 6))
        al = np.zeros(self.ngp); fl = np.zeros(self.ngp, np.uint8)
        rc = L.lib().pfem_get_state(self._ctx, ptr(U), ptr(tau), ptr(al), ptr(cpi), ptr(ep), ptr(fl, L._u8))
        check(rc, self._ctx)
        return dict(U=U, tau=tau, alpha=al, cpi=cpi, epsp=ep, flags=fl)

    @property
    def U(self):
        U = np.zeros(self.ndof)
        check(L.lib().pfem_get_state(self._ctx, ptr(U), None, None, None, None, None), self._ctx)
        return U

    def timer_start(self):
        check(L.lib().pfem_timer(self._ctx, 0, None), self._ctx)

    def timer_stop(self) -> float:
        ms = C.c_double()
        check(L.lib().pfem_timer(self._ctx, 1, C.byref(ms)), self._ctx)
        return ms.value

    # --- learned predictor (no counterpart in the reference) ---
    NPARAMS = 20752

    def mlp_init(self, seed=0):
        check(L.lib().pfem_mlp_init(self._ctx, int(seed)), self._ctx)

    def mlp_params(self, params=None):
        """Return the FP32 parameter vector, or load `params` (marks the predictor usable)."""
        if params is None:
            p = np.zeros(self.NPARAMS, np.float32)
            check(L.lib().pfem_mlp_params(self._ctx, 0, ptr(p, L._f), self.NPARAMS), self._ctx)
            return p
        p = np.ascontiguousarray(params, np.float32)
        check(L.lib().pfem_mlp_params(self._ctx, 1, ptr(p, L._f), self.NPARAMS), self._ctx)
        return p

    def mlp_forward(self, feats):
        f = np.ascontiguousarray(feats, np.float32)
        y = np.zeros((f.shape[0], 3), np.float32)
        check(L.lib().pfem_mlp_forward(self._ctx, ptr(f, L._f), f.shape[0], ptr(y, L._f)), self._ctx)
        return y

    def mlp_loss_grad(self, feats, targets):
        f = np.ascontiguousarray(feats, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        g = np.zeros(self.NPARAMS, np.float32)
        l = C.c_float()
        check(L.lib().pfem_mlp_loss_grad(self._ctx, ptr(f, L._f), ptr(t, L._f), f.shape[0], ptr(g, L._f),
                                         C.byref(l)), self._ctx)
        return l.value, g

    def mlp_record(self, op, capacity=0):
        n = C.c_int64()
        check(L.lib().pfem_mlp_record(self._ctx, {"start": 0, "stop": 1, "clear": 2, "size": 3}[op],
                                      int(capacity), C.byref(n)), self._ctx)
        return n.value

    def mlp_train(self, steps, batch=65536, lr=1e-3, seed=0):
        losses = np.zeros(steps, np.float32)
        check(L.lib().pfem_mlp_train(self._ctx, int(steps), int(batch), float(lr), int(seed), ptr(losses, L._f)),
              self._ctx)
        return losses

    def tangent_index_bytes(self) -> int:
        """Bytes per block column index the level-0 SpMV reads (2 or 4)."""
        b = C.c_int32()
        check(L.lib().pfem_tangent_index_bytes(self._ctx, C.byref(b)), self._ctx)
        return b.value

    def profile(self, what: int, reps: int = 10) -> float:
        ms = C.c_double()
        check(L.lib().pfem_profile(self._ctx, what, reps, C.byref(ms)), self._ctx)
        return ms.value


# ------------------------------------------------------------------ free functions
def fix(model, nodes, comp="all"):
    return model.fix(nodes, comp)


def prescribe(model, nodes, comp, value, ramp=True):
    return model.prescribe(nodes, comp, value, ramp)


def load(model, nodes, comp, value, distribute=False):
    return model.load(nodes, comp, value, distribute)


def solve(model, **kw) -> SolveResult:
    return model.solve(**kw)


def reset(model):
    return model.reset()


def nodal_displacements(model) -> np.ndarray:
    """nodal_displacements (Model.jl:169-178): 3 x nn, a view of the node-major
    displacement vector (the reference's column-major 3 x nn layout)."""
    return model.U.reshape(-1, 3).T


def gauss_kirchhoff(model) -> np.ndarray:
    """Committed Kirchhoff stress, 6 x ngp (Model.jl:227); a view of the per-GP
    (ngp, 6) array the library fills."""
    t = np.zeros((model.ngp, 6))
    check(L.lib().pfem_get_state(model._ctx, None, ptr(t), None, None, None, None), model._ctx)
    return t.T


def gauss_stress(model) -> np.ndarray:
    """Cauchy stress tau / det F (standard F), 6 x ngp (Model.jl:188-208)."""
    s = np.zeros((model.ngp, 6))
    check(L.lib().pfem_gauss_stress(model._ctx, ptr(s)), model._ctx)
    return s.T


def equivalent_plastic_strain(model) -> np.ndarray:
    """Committed equivalent plastic strain alpha per GP (Model.jl:232)."""
    a = np.zeros(model.ngp)
    check(L.lib().pfem_get_state(model._ctx, None, None, ptr(a), None, None, None), model._ctx)
    return a
