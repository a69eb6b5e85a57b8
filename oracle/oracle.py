"""CPU FP64 oracle for the finite-strain F-bar J2 path -- TEST INFRASTRUCTURE.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s ``cpu_baseline``
leg import this module, and only as the checker / the timed CPU baseline.  The
product library never links or calls it.

The arithmetic lives in ``pfem_oracle.cpp`` (a literal C++ restatement of
``lagrangian/src/{Materials,FiniteStrain,Elements,Assembly,BoundaryConditions}.jl``);
this file restates the driver logic of ``lagrangian/src/Solver.jl`` (``solve!``
:419-475, ``newton!`` :317-389, ``_freeze_bcs`` :192-218) and the
post-processing of ``lagrangian/src/Model.jl`` (``gauss_stress`` :188-208).

Linear solve: the reference sends the F-bar tangent to UMFPACK LU
(``Solver.jl:183-187, :237-240``); here SuperLU (``scipy.sparse.linalg.splu``)
stands in for it -- both are exact sparse LU, so Newton iterates agree to
rounding.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libpfem_oracle.so")
_lib = None

_d = C.POINTER(C.c_double)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)


def build() -> str:
    """Compile the oracle shared library with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        L.or_return_map.restype = C.c_int
        L.or_return_map.argtypes = [_d, _d, _d, _d, C.c_double, _d, _d, _d, _d, _d]
        L.or_finite_update.restype = C.c_int
        L.or_finite_update.argtypes = [_d, _d, _d, C.c_double, _d, _d, _d, _d, _d, _d, _d, _d]
        L.or_element.restype = C.c_int
        L.or_element.argtypes = [C.c_int, _d, C.c_double, _d, _d, _d, _d, _d, _d, _d, _d, _d,
                                 _d, _d, _d, _u8, _d]
        L.or_pattern_nnz.restype = C.c_int64
        L.or_pattern_nnz.argtypes = [C.c_int64, C.c_int64, _i64]
        L.or_pattern_fill.restype = None
        L.or_pattern_fill.argtypes = [C.c_int64, C.c_int64, _i64, _i64, _i64]
        L.or_element_colors.restype = C.c_int
        L.or_element_colors.argtypes = [C.c_int64, C.c_int64, _d, _i64]
        L.or_assemble.restype = C.c_int
        L.or_assemble.argtypes = [C.c_int, _d, _d, C.c_int64, C.c_int64, _d, _i64, _i64, _i64,
                                  _d, _d, _d, _d, _d, C.c_int, _d, _d, _d, _u8, C.c_int, _i64,
                                  C.POINTER(C.c_int), _d]
        L.or_impose_dirichlet.restype = None
        L.or_impose_dirichlet.argtypes = [C.c_int64, _i64, _i64, _d, _d, C.c_int64, _i64, _d,
                                          C.c_int, C.c_double, _d]
        _lib = L
    return _lib


def _p(a, t=_d):
    return a.ctypes.data_as(t) if a is not None else None


def _mat7(mat) -> np.ndarray:
    return np.array([mat.E, mat.nu, mat.sigy0, mat.Hiso, mat.Hkin, mat.sigsat_value, mat.delta],
                    dtype=np.float64)


@dataclass
class J2Material:
    """J2Material (Materials.jl:68-108): linear or saturation (Voce) isotropic
    hardening, sigma_y(a) = sigy0 + (sigsat - sigy0)(1 - exp(-delta a)) + Hiso a
    (yield_stress, :117-118), plus linear kinematic hardening Hkin."""
    E: float
    nu: float
    sigy0: float
    Hiso: float = 0.0
    Hkin: float = 0.0
    sigsat: float | None = None   # keyword default sigsat = sigy0
    delta: float = 0.0

    @property
    def sigsat_value(self):
        return self.sigy0 if self.sigsat is None else self.sigsat

    def yield_stress(self, a):
        return self.sigy0 + (self.sigsat_value - self.sigy0) * (1 - np.exp(-self.delta * a)) + self.Hiso * a

    def yield_slope(self, a):
        return self.delta * (self.sigsat_value - self.sigy0) * np.exp(-self.delta * a) + self.Hiso

    @property
    def G(self):
        return self.E / (2 * (1 + self.nu))

    @property
    def lam(self):
        return self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))

    def cmat(self) -> np.ndarray:
        a = self.lam + 2 * self.G
        Cm = np.zeros((6, 6))
        Cm[:3, :3] = self.lam
        Cm[0, 0] = Cm[1, 1] = Cm[2, 2] = a
        Cm[3, 3] = Cm[4, 4] = Cm[5, 5] = self.G
        return Cm


# ---------------------------------------------------------------- point level
def return_map(mat, eps, epsp=None, beta=None, alpha=0.0):
    """return_map (Materials.jl:159-250). Returns (sig, epsp, beta, alpha, D, plastic)."""
    eps = np.ascontiguousarray(eps, dtype=np.float64)
    epsp = np.zeros(6) if epsp is None else np.ascontiguousarray(epsp, dtype=np.float64)
    beta = np.zeros(6) if beta is None else np.ascontiguousarray(beta, dtype=np.float64)
    sig, ep2, b2, D = np.zeros(6), np.zeros(6), np.zeros(6), np.zeros(36)
    a2 = C.c_double(0.0)
    m7 = _mat7(mat)
    pl = lib().or_return_map(_p(m7), _p(eps), _p(epsp), _p(beta), alpha, _p(sig), _p(ep2),
                             _p(b2), C.byref(a2), _p(D))
    return sig, ep2, b2, a2.value, D.reshape(6, 6), pl


def finite_update(mat, F, cpi=None, alpha=0.0, beta=None):
    """finite_kinematics + finite_stress_update (+ dPdF), FiniteStrain.jl.

    F is a 3x3 array, beta the committed back stress in the reference
    configuration (None = 0).  Returns dict(tau, cpi_new, alpha, beta, epsp_inc,
    D, A, plastic) or raises ValueError when det F <= 0."""
    F9 = np.ascontiguousarray(np.asarray(F, dtype=np.float64).T.reshape(9))
    cpi = np.array([1, 1, 1, 0, 0, 0.0]) if cpi is None else np.ascontiguousarray(cpi, np.float64)
    beta = np.zeros(6) if beta is None else np.ascontiguousarray(beta, np.float64)
    tau, cn, bn, ei, D, A = (np.zeros(6), np.zeros(6), np.zeros(6), np.zeros(6), np.zeros(36),
                             np.zeros(81))
    a2 = C.c_double(0.0)
    m7 = _mat7(mat)
    st = lib().or_finite_update(_p(m7), _p(F9), _p(cpi), alpha, _p(beta), _p(tau), _p(cn),
                                C.byref(a2), _p(bn), _p(ei), _p(D), _p(A))
    if st < 0:
        raise ValueError("det F <= 0")
    return dict(tau=tau, cpi_new=cn, alpha=a2.value, beta=bn, epsp_inc=ei, D=D.reshape(6, 6),
                A=A.reshape(9, 9), plastic=st)


def element(fbar, mat, Xe, ue, cpi=None, alpha=None, sigy0=None, beta=None):
    """One Hex8 element: fbar 0 / 1 finite strain without / with F-bar
    (Elements.jl:405-494), 2 small strain (Elements.jl:323-360; cpi is then eps_p,
    tau is sigma).  Xe (8,3), ue (24,).  Returns dict."""
    Xe = np.ascontiguousarray(np.asarray(Xe, np.float64).reshape(24))
    ue = np.ascontiguousarray(np.asarray(ue, np.float64).reshape(24))
    if cpi is None:
        cpi = np.zeros(48) if int(fbar) == 2 else np.tile([1, 1, 1, 0, 0, 0.0], 8)
    cpi = np.ascontiguousarray(np.asarray(cpi, np.float64).reshape(48))
    alpha = np.zeros(8) if alpha is None else np.ascontiguousarray(alpha, np.float64)
    beta = np.zeros(48) if beta is None else np.ascontiguousarray(np.asarray(beta, np.float64).reshape(48))
    Fe, Ke, tau, cn, an, bn, ei = (np.zeros(24), np.zeros(576), np.zeros(48), np.zeros(48),
                                   np.zeros(8), np.zeros(48), np.zeros(48))
    fl = np.zeros(8, np.uint8)
    bJ = C.c_double(0.0)
    m7 = _mat7(mat)
    sy = mat.sigy0 if sigy0 is None else sigy0
    st = lib().or_element(int(fbar), _p(m7), sy, _p(Xe), _p(ue), _p(cpi), _p(alpha), _p(beta),
                          _p(Fe), _p(Ke), _p(tau), _p(cn), _p(an), _p(bn), _p(ei), _p(fl, _u8),
                          C.byref(bJ))
    if st < 0:
        raise ElementInversionError(1, -st, bJ.value)
    return dict(Fe=Fe, Ke=Ke.reshape(24, 24), tau=tau.reshape(8, 6), cpi_new=cn.reshape(8, 6),
                alpha=an, beta=bn.reshape(8, 6), epsp_inc=ei.reshape(8, 6), flags=fl)


class ElementInversionError(Exception):
    """ElementInversionError(e, g, J) (FiniteStrain.jl:42-52)."""

    def __init__(self, e, g, J):
        super().__init__(f"element {e}, Gauss point {g} is inverted (det F = J = {J} <= 0)")
        self.e, self.g, self.J = e, g, J


# ---------------------------------------------------------------- mesh level
def box_mesh(lx, ly, lz, nx, ny, nz):
    """box_mesh (Mesh.jl:30-59): nodes (3, nn) column-major, elements (8, ne) 1-based."""
    npx, npy = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    nodes = np.stack([lx * i.ravel() / nx, ly * j.ravel() / ny, lz * k.ravel() / nz]).astype(np.float64)
    ke, je, ie = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ie, je, ke = ie.ravel(), je.ravel(), ke.ravel()

    def nid(i, j, k):
        return (k * npy + j) * npx + i + 1

    elems = np.stack([nid(ie, je, ke), nid(ie + 1, je, ke), nid(ie + 1, je + 1, ke),
                      nid(ie, je + 1, ke), nid(ie, je, ke + 1), nid(ie + 1, je, ke + 1),
                      nid(ie + 1, je + 1, ke + 1), nid(ie, je + 1, ke + 1)]).astype(np.int64)
    return nodes, elems


def pattern(nn, elems):
    """build_sparsity pattern (Assembly.jl:99-146): 1-based colptr, rowval (int64)."""
    el = np.ascontiguousarray(elems.T, dtype=np.int64)  # (ne, 8) -> e*8+a
    ne = el.shape[0]
    nnz = lib().or_pattern_nnz(nn, ne, _p(el, _i64))
    colptr = np.zeros(3 * nn + 1, np.int64)
    rowval = np.zeros(nnz, np.int64)
    lib().or_pattern_fill(nn, ne, _p(el, _i64), _p(colptr, _i64), _p(rowval, _i64))
    return colptr, rowval


def box_nd_dofs(nx, ny, nz, leaf=64):
    """A nested-dissection order of the dofs of an (nx+1)(ny+1)(nz+1)-node box grid
    numbered i fastest (box_mesh, Mesh.jl:30-59): split the longest index range at
    its middle plane, order both halves recursively, the separator plane last.
    Any fill-reducing order leaves an exact LU's solution unchanged to rounding; this
    one keeps SuperLU's fill near the nested-dissection bound on box meshes, where its
    own orderings (COLAMD, MMD) fill 2-4x more."""
    npx, npy = nx + 1, ny + 1
    out = []

    def rec(i0, i1, j0, j1, k0, k1):
        di, dj, dk = i1 - i0, j1 - j0, k1 - k0
        if di <= 0 or dj <= 0 or dk <= 0:
            return
        if di * dj * dk <= leaf or max(di, dj, dk) < 3:
            k, j, i = np.meshgrid(np.arange(k0, k1), np.arange(j0, j1), np.arange(i0, i1), indexing="ij")
            out.append(((k * npy + j) * npx + i).ravel())
            return
        if di >= dj and di >= dk:
            m = (i0 + i1) // 2
            rec(i0, m, j0, j1, k0, k1); rec(m + 1, i1, j0, j1, k0, k1); rec(m, m + 1, j0, j1, k0, k1)
        elif dj >= dk:
            m = (j0 + j1) // 2
            rec(i0, i1, j0, m, k0, k1); rec(i0, i1, m + 1, j1, k0, k1); rec(i0, i1, m, m + 1, k0, k1)
        else:
            m = (k0 + k1) // 2
            rec(i0, i1, j0, j1, k0, m); rec(i0, i1, j0, j1, m + 1, k1); rec(i0, i1, j0, j1, m, m + 1)

    rec(0, nx + 1, 0, ny + 1, 0, nz + 1)
    pn = np.concatenate(out)
    return (3 * pn[:, None] + np.arange(3)[None, :]).ravel()


def nd_lu_solver(perm, stats=None):
    """linsolve(K, b) for OracleModel.newton: sparse LU (SuperLU, standing in for
    the reference's UMFPACK, Solver.jl:237-240) of K in the symmetric order `perm`.
    `stats`, a dict, collects the factorisation count and seconds."""
    import time

    def solve(K, b):
        t0 = time.perf_counter()
        Kp = K.tocsc()[perm][:, perm].tocsc()
        lu = spla.splu(Kp, permc_spec="NATURAL", diag_pivot_thresh=0.01, options=dict(SymmetricMode=True))
        x = np.empty_like(b)
        x[perm] = lu.solve(b[perm])
        if stats is not None:
            stats["lu"] = stats.get("lu", 0) + 1
            stats["lu_s"] = stats.get("lu_s", 0.0) + time.perf_counter() - t0
        return x
    return solve


def element_colors(nodes, elems):
    """element_colors (Assembly.jl:172-206) as a 0-based color id per element."""
    nn, ne = nodes.shape[1], elems.shape[1]
    nd = np.ascontiguousarray(nodes.T)
    col = np.zeros(ne, np.int64)
    nc = lib().or_element_colors(nn, ne, _p(nd), _p(col, _i64))
    return nc, col


# ---------------------------------------------------------------- model
@dataclass
class OracleModel:
    """Model (Model.jl:32-75) restated for the F-bar / finite / small-strain kinds."""
    nodes: np.ndarray            # (3, nn)
    elems: np.ndarray            # (8, ne) 1-based
    mat: J2Material
    fbar: bool = True
    small: bool = False          # small-strain kind (Elements.jl:323-360); fbar is then ignored
    sigy0_e: np.ndarray | None = None
    nthreads: int = 0
    dir_dofs: list = field(default_factory=list)
    dir_vals: list = field(default_factory=list)
    dir_ramp: list = field(default_factory=list)
    neu_dofs: list = field(default_factory=list)
    neu_vals: list = field(default_factory=list)

    def __post_init__(self):
        self.nn = self.nodes.shape[1]
        self.ne = self.elems.shape[1]
        self.ndof = 3 * self.nn
        self.colptr, self.rowval = pattern(self.nn, self.elems)
        self._nodes_rm = np.ascontiguousarray(self.nodes.T)
        self._el_rm = np.ascontiguousarray(self.elems.T, dtype=np.int64)
        if self.sigy0_e is not None:
            self.sigy0_e = np.ascontiguousarray(self.sigy0_e, np.float64)
        self.reset()

    # --- BC builders (Model.jl:102-145); comp in {'x','y','z','all'} ---
    @staticmethod
    def _comps(comp):
        return {"x": (1,), "y": (2,), "z": (3,), "all": (1, 2, 3)}[comp]

    def fix(self, nodes, comp="all"):
        for n in nodes:
            for c in self._comps(comp):
                self.dir_dofs.append(3 * (int(n) - 1) + c)
                self.dir_vals.append(0.0)
                self.dir_ramp.append(False)

    def prescribe(self, nodes, comp, value, ramp=True):
        for n in nodes:
            for c in self._comps(comp):
                self.dir_dofs.append(3 * (int(n) - 1) + c)
                self.dir_vals.append(float(value))
                self.dir_ramp.append(bool(ramp))

    def load(self, nodes, comp, value, distribute=False):
        per = float(value) / len(nodes) if distribute else float(value)
        for n in nodes:
            for c in self._comps(comp):
                self.neu_dofs.append(3 * (int(n) - 1) + c)
                self.neu_vals.append(per)

    def reset(self):
        ngp = 8 * self.ne
        self.U = np.zeros(self.ndof)
        self.cpi = np.zeros((ngp, 6))    # Cp^-1 (finite kinds) or eps_p (small strain)
        if not self.small:
            self.cpi[:, :3] = 1.0
        self.alpha = np.zeros(ngp)
        self.beta = np.zeros((ngp, 6))   # back stress (reference configuration for the finite kinds)
        self.epsp = np.zeros((ngp, 6))
        self.tau = np.zeros((ngp, 6))
        self.flags = np.zeros(ngp, np.uint8)

    # --- assembly (Assembly.jl:238-331) ---
    def assemble(self, U, commit=False, cpi=None, alpha=None):
        nnz = len(self.rowval)
        nz = np.zeros(nnz)
        R = np.zeros(self.ndof)
        tau = np.zeros((8 * self.ne, 6))
        fl = np.zeros(8 * self.ne, np.uint8)
        cpi = self.cpi if cpi is None else cpi
        alpha = self.alpha if alpha is None else alpha
        be = C.c_int64(0); bg = C.c_int(0); bJ = C.c_double(0)
        U = np.ascontiguousarray(U, np.float64)
        m7 = _mat7(self.mat)
        st = lib().or_assemble(2 if self.small else int(self.fbar), _p(m7), _p(self.sigy0_e), self.nn, self.ne,
                               _p(self._nodes_rm), _p(self._el_rm, _i64), _p(self.colptr, _i64),
                               _p(self.rowval, _i64), _p(U), _p(cpi), _p(alpha),
                               _p(self.epsp), _p(self.beta) if self.mat.Hkin > 0 else None,
                               int(commit), _p(nz), _p(R), _p(tau),
                               _p(fl, _u8), self.nthreads, C.byref(be), C.byref(bg), C.byref(bJ))
        if st < 0:
            raise ElementInversionError(be.value, bg.value, bJ.value)
        K = sp.csc_matrix((nz, self.rowval - 1, self.colptr - 1), shape=(self.ndof, self.ndof))
        return K, R, tau, fl

    def freeze_bcs(self):
        """_freeze_bcs (Solver.jl:192-218): dedupe per dof, last wins."""
        last = {}
        for d, v, r in zip(self.dir_dofs, self.dir_vals, self.dir_ramp):
            last[d] = (v, r)
        rd = [d for d, (v, r) in last.items() if r]
        rv = [v for d, (v, r) in last.items() if r]
        fd = [d for d, (v, r) in last.items() if not r]
        fv = [v for d, (v, r) in last.items() if not r]
        return ((np.array(rd, np.int64), np.array(rv, np.float64)),
                (np.array(fd, np.int64), np.array(fv, np.float64)))

    def impose(self, K, R, dofs, vals, ramp, lam, U):
        if len(dofs) == 0:
            return
        lib().or_impose_dirichlet(self.ndof, _p(self.colptr, _i64), _p(self.rowval, _i64),
                                  _p(K.data), _p(R), len(dofs), _p(dofs, _i64), _p(vals),
                                  int(ramp), lam, _p(np.ascontiguousarray(U)))

    def fext(self, lam):
        F = np.zeros(self.ndof)
        for d, v in zip(self.neu_dofs, self.neu_vals):
            F[d - 1] += lam * v
        return F

    def _residual(self, lam, ramp_set, fix_set, Fext):
        K, R, tau, fl = self.assemble(self.U)
        R -= Fext
        self.impose(K, R, ramp_set[0], ramp_set[1], True, lam, self.U)
        self.impose(K, R, fix_set[0], fix_set[1], False, lam, self.U)
        return K, R

    def newton(self, lam, ramp_set, fix_set, tol, maxiter, linsolve=None, line_search=False):
        """newton! (Solver.jl:317-389) with exact sparse LU.  line_search=True adds
        the same backtracking globalisation as the GPU path (halve the step, at
        most 8 times, until the imposed residual norm decreases)."""
        Fext = self.fext(lam)
        fext_norm = float(np.sqrt(np.sum(Fext ** 2)))
        hist = []
        ref = 1.0
        conv = False
        K, R = self._residual(lam, ramp_set, fix_set, Fext)
        rnorm = float(np.linalg.norm(R))
        for it in range(1, maxiter + 1):
            hist.append(rnorm)
            if it == 1:
                ref = max(rnorm, fext_norm, 1.0)
            if rnorm <= tol * ref:
                conv = True
                break
            if it == maxiter:
                break
            b = -R
            dU = spla.splu(K.tocsc()).solve(b) if linsolve is None else linsolve(K, b)
            U0 = self.U.copy()
            a = 1.0
            for bt in range(9):
                self.U = U0 + a * dU
                try:
                    K2, R2 = self._residual(lam, ramp_set, fix_set, Fext)
                    r2 = float(np.linalg.norm(R2))
                except ElementInversionError:
                    if not line_search or bt >= 8:
                        raise
                    r2 = np.inf
                if not line_search or (np.isfinite(r2) and (r2 < (1 - 1e-4 * a) * rnorm or bt >= 8)):
                    break
                a *= 0.5
            K, R, rnorm = K2, R2, r2
        return conv, hist

    def solve(self, nsteps=10, tol=1e-8, maxiter=25, linsolve=None, step_callback=None,
              line_search=False):
        """solve! (Solver.jl:419-475).  Returns dict(converged, iters, residuals)."""
        self.reset()
        ramp_set, fix_set = self.freeze_bcs()
        iters, resid = [], []
        allconv = True
        for n in range(1, nsteps + 1):
            lam = n / nsteps
            conv, hist = self.newton(lam, ramp_set, fix_set, tol, maxiter, linsolve, line_search)
            iters.append(len(hist)); resid.append(hist)
            if not conv:
                allconv = False
                break
            # commit: re-assemble with commit=true (Solver.jl:470-471)
            _, _, tau, fl = self.assemble(self.U, commit=True)
            self.tau, self.flags = tau, fl
            if step_callback is not None:
                step_callback(n, self)
        return dict(converged=allconv, iters=iters, residuals=resid)

    # --- post-processing (Model.jl:169-232) ---
    def nodal_displacements(self):
        return self.U.reshape(-1, 3).T.copy()

    def gauss_stress(self):
        """Cauchy = tau / det F_gp (standard F, not F-bar), Model.jl:188-208; the
        small-strain kind stores sigma itself."""
        if self.small:
            return self.tau.copy()
        from_gp = np.zeros_like(self.tau)
        detF = gp_detF(self.nodes, self.elems, self.U)
        invJ = np.where(detF > 0, 1.0 / np.where(detF > 0, detF, 1.0), 1.0)
        from_gp[:] = self.tau * invJ[:, None]
        return from_gp

    def equivalent_plastic_strain(self):
        return self.alpha.copy()


_G = 1.0 / np.sqrt(3.0)
_GSGN = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float64)


def _dshape(xi):
    nat = _GSGN  # node natural coords share the Gauss-point sign table
    dN = np.zeros((8, 3))
    dN[:, 0] = 0.125 * nat[:, 0] * (1 + nat[:, 1] * xi[1]) * (1 + nat[:, 2] * xi[2])
    dN[:, 1] = 0.125 * nat[:, 1] * (1 + nat[:, 0] * xi[0]) * (1 + nat[:, 2] * xi[2])
    dN[:, 2] = 0.125 * nat[:, 2] * (1 + nat[:, 0] * xi[0]) * (1 + nat[:, 1] * xi[1])
    return dN


def gp_detF(nodes, elems, U):
    """det F at every Gauss point (standard F), vectorised over elements."""
    Xe = nodes.T[elems.T - 1]                      # (ne, 8, 3)
    ue = U.reshape(-1, 3)[elems.T - 1]             # (ne, 8, 3)
    out = np.zeros((elems.shape[1], 8))
    for g in range(8):
        dN = _dshape(_GSGN[g] * _G)                # (8, 3)
        J = np.einsum("eai,aj->eij", Xe, dN)
        dNdX = np.einsum("am,emj->eaj", dN, np.linalg.inv(J))
        F = np.eye(3)[None] + np.einsum("eai,eaj->eij", ue, dNdX)
        out[:, g] = np.linalg.det(F)
    return out.reshape(-1)
