"""Seeded synthetic workloads with the shapes of the headline configurations.

No public dataset is involved: meshes, geometric noise, yield-stress fields and
boundary conditions are generated here from seeds, and the same arrays feed the
GPU path and the CPU oracle.  Units: mm, MPa, N.

Boundary-condition notes.  Two of the configurations leave rigid-body modes
free as literally stated (a bottom face with only uz fixed leaves x/y
translation and the z rotation free; the corner-pinned cube leaves the z
rotation free); the direct LU of the reference would be singular there.  They
receive a minimal 3-2-1 constraint -- node (0,0,0): ux = uy = 0, node (1,0,0):
uy = 0 -- which removes only rigid motion and changes no stress.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .model import Mesh, box_mesh

SEED = 20261203
MAT = dict(E=200e3, nu=0.3, sigy0=250.0, Hiso=2000.0, Hkin=0.0)


@dataclass
class Workload:
    name: str
    mesh: Mesh
    material: dict
    sigy0_e: np.ndarray | None
    dir_dofs: np.ndarray          # 1-based
    dir_vals: np.ndarray
    dir_ramp: np.ndarray          # uint8
    nsteps: int
    tol: float
    neu_dofs: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    neu_vals: np.ndarray = field(default_factory=lambda: np.zeros(0))
    meta: dict = field(default_factory=dict)

    def apply(self, model):
        """Push the BCs into a Model: arrays for the product model, lists for the
        oracle's (whose builders append)."""
        conv = (lambda a, t: np.array(a, t)) if hasattr(model, "_bcs_dirty") else (lambda a, t: np.array(a, t).tolist())
        model.dir_dofs = conv(self.dir_dofs, np.int64)
        model.dir_vals = conv(self.dir_vals, np.float64)
        model.dir_ramp = conv(self.dir_ramp, np.uint8)
        model.neu_dofs = conv(self.neu_dofs, np.int64)
        model.neu_vals = conv(self.neu_vals, np.float64)
        if hasattr(model, "_bcs_dirty"):
            model._bcs_dirty = True
        return model


class _BC:
    def __init__(self):
        self.d, self.v, self.r = [], [], []

    def add(self, nodes, comps, value, ramp):
        for n in np.atleast_1d(nodes):
            for c in comps:
                self.d.append(3 * (int(n) - 1) + c); self.v.append(float(value)); self.r.append(1 if ramp else 0)

    def arrays(self):
        return np.array(self.d, np.int64), np.array(self.v, np.float64), np.array(self.r, np.uint8)


def _near(a, b, tol=1e-9):
    return np.abs(a - b) <= tol


def _node_at(mesh, x, y, z):
    X = mesh.nodes
    idx = np.nonzero(_near(X[0], x) & _near(X[1], y) & _near(X[2], z))[0]
    return idx + 1


def jitter_interior(mesh: Mesh, h, frac, rng) -> Mesh:
    """Perturb every node not on the bounding box by U(-frac h, frac h) per axis."""
    X = mesh.nodes.copy()
    lo, hi = X.min(1, keepdims=True), X.max(1, keepdims=True)
    interior = np.all((X > lo + 1e-9) & (X < hi - 1e-9), axis=0)
    X[:, interior] += rng.uniform(-frac * h, frac * h, size=(3, int(interior.sum())))
    return Mesh(X, mesh.elements)


def lognormal_sigy(ne, mean, cov, rng):
    s = np.sqrt(np.log(1.0 + cov * cov))
    return np.exp(rng.normal(np.log(mean) - 0.5 * s * s, s, size=ne))


def config0(n=8, nsteps=10, tol=1e-10) -> Workload:
    """Unit cube n^3, uz = 0 on z = 0 with corner (0,0,0) pinned, top uz = 0.05 ramped."""
    m = box_mesh(1, 1, 1, n, n, n)
    bc = _BC()
    z0 = np.nonzero(_near(m.nodes[2], 0.0))[0] + 1
    z1 = np.nonzero(_near(m.nodes[2], 1.0))[0] + 1
    bc.add(z0, (3,), 0.0, False)
    bc.add(_node_at(m, 0, 0, 0), (1, 2, 3), 0.0, False)
    bc.add(_node_at(m, 1, 0, 0), (2,), 0.0, False)     # 3-2-1: removes the z rotation
    bc.add(z1, (3,), 0.05, True)
    d, v, r = bc.arrays()
    return Workload(f"cube{n}_tension", m, dict(MAT), None, d, v, r, nsteps, tol,
                    meta=dict(config=0, n=n))


def config1(nx=80, ny=16, nz=16, nsteps=60, tol=1e-8, stretch=0.30) -> Workload:
    """Necking bar 10x2x2, sigma_y -2% in element layer i = nx/2, 30% stretch."""
    m = box_mesh(10.0, 2.0, 2.0, nx, ny, nz)
    ne = m.nelem
    i_of_e = np.arange(ne) % nx
    sy = np.full(ne, MAT["sigy0"])
    sy[i_of_e == nx // 2] *= 0.98
    bc = _BC()
    X = m.nodes
    bc.add(np.nonzero(_near(X[0], 0.0))[0] + 1, (1,), 0.0, False)
    bc.add(np.nonzero(_near(X[1], 0.0))[0] + 1, (2,), 0.0, False)
    bc.add(np.nonzero(_near(X[2], 0.0))[0] + 1, (3,), 0.0, False)
    bc.add(np.nonzero(_near(X[0], 10.0))[0] + 1, (1,), stretch * 10.0, True)
    d, v, r = bc.arrays()
    return Workload(f"bar{nx}x{ny}x{nz}_neck", m, dict(MAT), sy, d, v, r, nsteps, tol,
                    meta=dict(config=1, nx=nx, ny=ny, nz=nz))


def config2(n=64, nsteps=40, tol=1e-8, seed=SEED + 2, compress=0.2) -> Workload:
    """Unit cube n^3, interior nodes jittered +-10% h, lognormal sigma_y (CoV 0.1),
    bottom uz = 0, top uz = -compress ramped, 3-2-1 rigid-body constraint."""
    rng = np.random.default_rng(seed)
    m = jitter_interior(box_mesh(1, 1, 1, n, n, n), 1.0 / n, 0.1, rng)
    sy = lognormal_sigy(m.nelem, MAT["sigy0"], 0.1, rng)
    bc = _BC()
    X = m.nodes
    bc.add(np.nonzero(_near(X[2], 0.0))[0] + 1, (3,), 0.0, False)
    bc.add(np.nonzero(_near(X[2], 1.0))[0] + 1, (3,), -compress, True)
    bc.add(_node_at(m, 0, 0, 0), (1, 2), 0.0, False)
    bc.add(_node_at(m, 1, 0, 0), (2,), 0.0, False)
    d, v, r = bc.arrays()
    return Workload(f"cube{n}_jitter_compress", m, dict(MAT), sy, d, v, r, nsteps, tol,
                    meta=dict(config=2, n=n, seed=seed))


def config3(n=150, nsteps=30, tol=1e-8, seed=SEED + 3, patch=30, depth=0.1) -> Workload:
    """Unit cube n^3 (jitter + lognormal field as config 2), bottom clamped, a central
    patch x patch node square of the top face indented by `depth` (ramped)."""
    rng = np.random.default_rng(seed)
    m = jitter_interior(box_mesh(1, 1, 1, n, n, n), 1.0 / n, 0.1, rng)
    sy = lognormal_sigy(m.nelem, MAT["sigy0"], 0.1, rng)
    bc = _BC()
    X = m.nodes
    bc.add(np.nonzero(_near(X[2], 0.0))[0] + 1, (1, 2, 3), 0.0, False)
    top = np.nonzero(_near(X[2], 1.0))[0]
    ii = np.rint(X[0, top] * n).astype(int)
    jj = np.rint(X[1, top] * n).astype(int)
    lo = (n + 1 - patch) // 2
    sel = top[(ii >= lo) & (ii < lo + patch) & (jj >= lo) & (jj < lo + patch)] + 1
    bc.add(sel, (3,), -depth, True)
    d, v, r = bc.arrays()
    return Workload(f"cube{n}_indent", m, dict(MAT), sy, d, v, r, nsteps, tol,
                    meta=dict(config=3, n=n, seed=seed, patch=patch))


def config4_path(n=32, nsteps=20, seed=SEED + 4, amp=0.05) -> Workload:
    """One learned-predictor training path: cube n^3, bottom clamped, top face driven by
    an affine displacement with 6 components ~ U(-amp, amp) (3 translations, 3 small
    rotations, scaled by the cube size)."""
    rng = np.random.default_rng(seed)
    m = box_mesh(1, 1, 1, n, n, n)
    c = rng.uniform(-amp, amp, size=6)
    bc = _BC()
    X = m.nodes
    bc.add(np.nonzero(_near(X[2], 0.0))[0] + 1, (1, 2, 3), 0.0, False)
    top = np.nonzero(_near(X[2], 1.0))[0]
    x, y, z = X[0, top] - 0.5, X[1, top] - 0.5, X[2, top]
    # small rotation vector (c3, c4, c5) about the top-face centre, plus translation
    ux = c[0] + (c[4] * (z - 1.0) - c[5] * y)
    uy = c[1] + (c[5] * x - c[3] * (z - 1.0))
    uz = c[2] + (c[3] * y - c[4] * x)
    for k, nidx in enumerate(top):
        bc.add([nidx + 1], (1,), ux[k], True)
        bc.add([nidx + 1], (2,), uy[k], True)
        bc.add([nidx + 1], (3,), uz[k], True)
    d, v, r = bc.arrays()
    return Workload(f"cube{n}_path{seed}", m, dict(MAT), None, d, v, r, nsteps, 1e-8,
                    meta=dict(config=4, n=n, seed=seed, coeffs=c.tolist()))


CONFIGS = {0: config0, 1: config1, 2: config2, 3: config3}
