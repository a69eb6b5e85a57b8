"""One-time topology built on the device (block pattern, rank table) against the
host build of a topology-only context: the same CSC pattern (Assembly.jl:99-162)
and colors, and an assembly that goes through the device-built rank table."""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu
MAT = P.J2Material(210e3, 0.3, 250.0, 1000.0)


def _meshes():
    yield "box", P.box_mesh(2.0, 1.0, 1.5, 7, 5, 3)
    yield "jittered", W.config2(n=6).mesh
    yield "necking_bar", W.config1(nx=12, ny=3, nz=3).mesh
    # 65 copies of one element: every node is in 65 elements, more than the
    # device kernel stages, so the host path builds this pattern
    box = P.box_mesh(1, 1, 1, 1, 1, 1)
    yield "stacked", P.Mesh(box.nodes, np.repeat(box.elements, 65, axis=1))


@pytest.mark.parametrize("name,mesh", list(_meshes()))
def test_device_pattern_matches_host(name, mesh):
    G = P.Model(mesh, MAT)
    H = P.Model(mesh, MAT, device=-1)
    cg, rg = G.pattern()
    ch, rh = H.pattern()
    assert np.array_equal(cg, ch) and np.array_equal(rg, rh), name
    assert G.colors()[0] == H.colors()[0] and np.array_equal(G.colors()[1], H.colors()[1]), name


def test_assembly_through_device_rank_table(oracle):
    w = W.config2(n=5)
    M = P.Model(w.mesh, P.J2Material(**w.material), element="finite_fbar", sigy0_e=w.sigy0_e)
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), sigy0_e=w.sigy0_e)
    rng = np.random.default_rng(3)
    U = 1e-3 * rng.standard_normal(M.ndof)
    K, R, _, _ = M.assemble(U)
    Ko, Ro, _, _ = om.assemble(U)
    assert abs(K - Ko.tocsr()).max() / abs(Ko).max() < 1e-10
    assert np.linalg.norm(R - Ro) / np.linalg.norm(Ro) < 1e-10
