"""The oracle's nested-dissection LU (used for the full-size necking-bar and 16^3
fixtures and the CPU baseline) is an exact solve: a permutation of the dofs and
the same solution as SuperLU in its own order."""
import numpy as np
import scipy.sparse.linalg as spla

from plasticity_b200 import workloads as W


def test_nd_order_is_a_permutation(oracle):
    for dims in ((3, 2, 2), (8, 3, 5), (6, 6, 6)):
        p = oracle.box_nd_dofs(*dims)
        nn = (dims[0] + 1) * (dims[1] + 1) * (dims[2] + 1)
        assert np.array_equal(np.sort(p), np.arange(3 * nn))


def test_nd_lu_matches_superlu(oracle):
    w = W.config2(n=6)
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), fbar=True,
                            sigy0_e=w.sigy0_e)
    w.apply(om)
    ramp, fix = om.freeze_bcs()
    K, R = om._residual(0.1, ramp, fix, om.fext(0.1))
    stats = {}
    x = oracle.nd_lu_solver(oracle.box_nd_dofs(6, 6, 6), stats)(K, -R)
    xr = spla.splu(K.tocsc()).solve(-R)
    assert np.linalg.norm(x - xr) <= 1e-12 * np.linalg.norm(xr)
    assert stats["lu"] == 1
