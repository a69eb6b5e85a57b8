"""Configuration 3 at its stated size: the 150^3 jittered / lognormal cube
(3,375,000 Hex8 F-bar elements, 10,328,853 DOF) with the central 30 x 30-node
top-face indentation.

- The assembly against the oracle on a sub-block: a 20^3-element block of the
  mesh is handed to the oracle as a mesh of its own (same nodes, committed state
  and yield stresses).  At every node whose eight elements all lie in the block
  the internal force is complete in both, so the GPU's full-mesh R must equal the
  oracle's there; Kirchhoff stress and flags of the block's Gauss points too.
  (The oracle's full 150^3 CSC tangent would need ~13 GB of host memory and
  minutes per assembly; the block covers the same arithmetic.)
- The first two increments of the load path, FP64 against mixed precision.
"""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu
N = 150


@pytest.fixture(scope="module")
def w():
    return W.config3(n=N)


def _model(w):
    M = P.Model(w.mesh, P.J2Material(**w.material), sigy0_e=w.sigy0_e)
    w.apply(M)
    return M


def test_config3_subblock_assembly_vs_oracle(w, oracle):
    M = _model(w)
    X = w.mesh.nodes
    rng = np.random.default_rng(3)
    U = (np.stack([0.00075 * (X[0] - 0.5), 0.0005 * (X[1] - 0.5), -0.001 * X[2]]).T.reshape(-1)
         + 2e-4 / N * rng.standard_normal(M.ndof))
    M.assemble(0.5 * U, commit=True)
    _, R, tau, fl = M.assemble(U, want_K=False)
    assert 0.05 < fl.mean() < 0.999

    lo, nb = 60, 20                                   # elements i, j, k in [60, 80)
    npx = N + 1
    ke, je, ie = np.meshgrid(np.arange(lo, lo + nb), np.arange(lo, lo + nb), np.arange(lo, lo + nb),
                             indexing="ij")
    eids = ((ke * N + je) * N + ie).ravel()           # 0-based element ids
    kn, jn, inn = np.meshgrid(np.arange(lo, lo + nb + 1), np.arange(lo, lo + nb + 1),
                              np.arange(lo, lo + nb + 1), indexing="ij")
    nids = ((kn * npx + jn) * npx + inn).ravel()      # 0-based node ids of the block
    local = np.full(M.nn, -1, np.int64)
    local[nids] = np.arange(len(nids))
    el = local[w.mesh.elements[:, eids] - 1] + 1       # 1-based in the block
    assert (el > 0).all()
    om = oracle.OracleModel(np.ascontiguousarray(X[:, nids]), el, oracle.J2Material(**w.material),
                            fbar=True, sigy0_e=w.sigy0_e[eids], nthreads=0)
    dofs = (3 * nids[:, None] + np.arange(3)[None, :]).ravel()
    om.assemble(0.5 * U[dofs], commit=True)
    Ko, Ro, tauo, flo = om.assemble(U[dofs])
    # nodes strictly inside the block: all eight elements belong to it
    inner = ((kn > lo) & (kn < lo + nb) & (jn > lo) & (jn < lo + nb) & (inn > lo) & (inn < lo + nb)).ravel()
    din = (3 * np.nonzero(inner)[0][:, None] + np.arange(3)[None, :]).ravel()
    Rg = R[dofs][din]
    assert np.linalg.norm(Rg - Ro[din]) <= 1e-10 * np.linalg.norm(Ro[din])
    gps = (8 * eids[:, None] + np.arange(8)[None, :]).ravel()
    assert np.abs(tau[gps] - tauo).max() <= 1e-10 * np.abs(tauo).max()
    assert np.array_equal(fl[gps], flo)


def test_config3_mixed_matches_fp64_first_increments(w):
    fp64 = _model(w)
    mixed = _model(w)
    for s in (1, 2):
        lam = s / w.nsteps
        fp64.newton(lam, tol=1e-10, maxiter=60, precision="fp64", predictor="extrapolate", line_search=True)
        mixed.newton(lam, tol=1e-10, maxiter=60, precision="mixed", predictor="extrapolate", line_search=True)
    Ut, Um = fp64.U, mixed.U
    assert np.linalg.norm(Um - Ut) / np.linalg.norm(Ut) < 1e-8
    at, am = P.equivalent_plastic_strain(fp64), P.equivalent_plastic_strain(mixed)
    assert np.abs(am - at).max() / max(np.abs(at).max(), 1e-300) < 1e-6
