"""The .vtu writer (Visualization.jl:129-205) on an oracle solution: the file
parses, carries the reference's arrays and names, and the cell fields are the
Gauss-point averages; the small strain equals the oracle's B u."""
import xml.etree.ElementTree as ET

import numpy as np

from plasticity_b200 import visualization as V
from plasticity_b200 import workloads as W


def _arrays(root):
    out = {}
    for da in root.iter("DataArray"):
        name = da.get("Name") or "Points"
        out[name] = (da, np.array(da.text.split(), dtype=float))
    return out


def test_write_vtu_arrays_roundtrip(oracle, tmp_path):
    w = W.config0(n=3, nsteps=2)
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), fbar=True)
    w.apply(om)
    assert om.solve(nsteps=2, tol=1e-10)["converged"]
    sig = om.gauss_stress()
    fn = V.write_vtu_arrays(str(tmp_path / "cube"), w.mesh.nodes, w.mesh.elements, om.U, sig, om.alpha)
    assert fn.endswith(".vtu")
    root = ET.parse(fn).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    nn, ne = w.mesh.nnodes, w.mesh.nelem
    assert int(piece.get("NumberOfPoints")) == nn and int(piece.get("NumberOfCells")) == ne
    A = _arrays(root)
    assert np.allclose(A["Points"][1].reshape(nn, 3), w.mesh.nodes.T)
    assert np.array_equal(A["connectivity"][1].reshape(ne, 8), w.mesh.elements.T - 1)
    assert np.array_equal(A["offsets"][1], 8 * np.arange(1, ne + 1))
    assert np.all(A["types"][1] == 12)
    assert np.allclose(A["Displacement"][1].reshape(nn, 3), om.U.reshape(nn, 3), rtol=0, atol=0)
    sc = sig.reshape(ne, 8, 6).mean(axis=1)
    assert np.allclose(A["Stress"][1].reshape(ne, 6), sc, rtol=1e-15, atol=0)
    assert [A["Stress"][0].get(f"ComponentName{i}") for i in range(6)] == ["xx", "yy", "zz", "xy", "yz", "zx"]
    vm = np.sqrt(0.5 * ((sc[:, 0] - sc[:, 1]) ** 2 + (sc[:, 1] - sc[:, 2]) ** 2 + (sc[:, 2] - sc[:, 0]) ** 2)
                 + 3 * (sc[:, 3] ** 2 + sc[:, 4] ** 2 + sc[:, 5] ** 2))
    assert np.allclose(A["VonMises"][1], vm, rtol=1e-14)
    assert np.allclose(A["MeanStress"][1], sc[:, :3].mean(axis=1), rtol=1e-14)
    assert np.allclose(A["EqPlasticStrain"][1], om.alpha.reshape(ne, 8).mean(axis=1), rtol=1e-14)
    # small strain B u against the oracle's small-strain element (its eps_p-free trial stress)
    eps = V.gauss_strain(w.mesh.nodes, w.mesh.elements, om.U)
    e0 = w.mesh.elements[:, 0] - 1
    Xe = w.mesh.nodes[:, e0].T
    ue = om.U.reshape(-1, 3)[e0].reshape(-1)
    big = oracle.J2Material(**{**w.material, "sigy0": 1e12})
    out = oracle.element(2, big, Xe, ue)             # elastic: sigma = C eps
    lam = big.E * big.nu / ((1 + big.nu) * (1 - 2 * big.nu)); G = big.E / (2 * (1 + big.nu))
    C = np.zeros((6, 6)); C[:3, :3] = lam; C[[0, 1, 2], [0, 1, 2]] += 2 * G; C[[3, 4, 5], [3, 4, 5]] = G
    assert np.allclose(eps[:8] @ C.T, out["tau"], rtol=1e-10, atol=1e-8)
