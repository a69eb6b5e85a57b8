"""VTK export (`.vtu`, ASCII XML unstructured grid) for ParaView / VisIt.

Restates lagrangian/src/Visualization.jl: the mesh with per-node displacements and
per-element (Gauss-point averaged) stress, strain, von Mises stress, mean stress and
equivalent plastic strain, written with the same array names, component names and
layout as the reference's `write_vtu` (Visualization.jl:129-205).
"""
from __future__ import annotations

import numpy as np

_VOIGT_NAMES = ("xx", "yy", "zz", "xy", "yz", "zx")
_GSGN = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float64)


def von_mises(sig):
    """von Mises stress of Voigt stresses (..., 6), physical shears (Visualization.jl:28-33)."""
    s = np.asarray(sig, np.float64)
    sxx, syy, szz, sxy, syz, szx = (s[..., i] for i in range(6))
    return np.sqrt(0.5 * ((sxx - syy) ** 2 + (syy - szz) ** 2 + (szz - sxx) ** 2)
                   + 3.0 * (sxy ** 2 + syz ** 2 + szx ** 2))


def gauss_strain(nodes, elements, U, chunk=65536):
    """Small strain eps = B u_e at every Gauss point, engineering-shear Voigt,
    shape (ngp, 6) with gp = 8 e + g (gauss_strain, Visualization.jl:43-58).
    nodes (3, nn), elements (8, ne) 1-based, U (3 nn,)."""
    X = np.asarray(nodes, np.float64).T
    E = np.asarray(elements, np.int64).T - 1
    Un = np.asarray(U, np.float64).reshape(-1, 3)
    ne = E.shape[0]
    gc = 1.0 / np.sqrt(3.0)
    # dN/dxi at the 8 Gauss points: (8 gp, 8 nodes, 3)
    xi = _GSGN * gc
    dN = np.empty((8, 8, 3))
    for g in range(8):
        x, y, z = xi[g]
        dN[g, :, 0] = 0.125 * _GSGN[:, 0] * (1 + _GSGN[:, 1] * y) * (1 + _GSGN[:, 2] * z)
        dN[g, :, 1] = 0.125 * _GSGN[:, 1] * (1 + _GSGN[:, 0] * x) * (1 + _GSGN[:, 2] * z)
        dN[g, :, 2] = 0.125 * _GSGN[:, 2] * (1 + _GSGN[:, 0] * x) * (1 + _GSGN[:, 1] * y)
    out = np.empty((ne, 8, 6))
    for a in range(0, ne, chunk):
        b = min(ne, a + chunk)
        Xe = X[E[a:b]]                                   # (m, 8, 3)
        ue = Un[E[a:b]]                                  # (m, 8, 3)
        J = np.einsum("ani,gnj->gaij", Xe, dN)           # (8, m, 3, 3): J_ij = sum_n X_ni dN_nj
        Ji = np.linalg.inv(J)
        dNdX = np.einsum("gnk,gakj->ganj", dN, Ji)       # (8, m, 8, 3)
        H = np.einsum("ani,ganj->gaij", ue, dNdX)        # displacement gradient (8, m, 3, 3)
        eps = np.stack([H[..., 0, 0], H[..., 1, 1], H[..., 2, 2],
                        H[..., 0, 1] + H[..., 1, 0], H[..., 1, 2] + H[..., 2, 1],
                        H[..., 2, 0] + H[..., 0, 2]], axis=-1)
        out[a:b] = np.transpose(eps, (1, 0, 2))
    return out.reshape(-1, 6)


def _fmt(a):
    return "\n".join("          " + " ".join(repr(float(v)) for v in row) for row in np.atleast_2d(a))


def write_vtu_arrays(filename, nodes, elements, U, sigma_gp, alpha_gp):
    """Write the `.vtu` file from arrays: nodes (3, nn), elements (8, ne) 1-based,
    U (3 nn,), Gauss-point stress (ngp, 6) and equivalent plastic strain (ngp,).
    Returns the path written (`.vtu` appended when missing)."""
    fn = filename if str(filename).endswith(".vtu") else f"{filename}.vtu"
    nodes = np.asarray(nodes, np.float64)
    elements = np.asarray(elements, np.int64)
    nn, ne = nodes.shape[1], elements.shape[1]
    sig_c = np.asarray(sigma_gp, np.float64).reshape(ne, 8, 6).mean(axis=1)
    eps_c = gauss_strain(nodes, elements, U).reshape(ne, 8, 6).mean(axis=1)
    alp_c = np.asarray(alpha_gp, np.float64).reshape(ne, 8).mean(axis=1)
    Un = np.asarray(U, np.float64).reshape(nn, 3)
    comps = " ".join(f'ComponentName{i}="{n}"' for i, n in enumerate(_VOIGT_NAMES))
    with open(fn, "w") as f:
        w = f.write
        w('<?xml version="1.0"?>\n')
        w('<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian">\n')
        w("  <UnstructuredGrid>\n")
        w(f'    <Piece NumberOfPoints="{nn}" NumberOfCells="{ne}">\n')
        w("      <Points>\n")
        w('        <DataArray type="Float64" NumberOfComponents="3" format="ascii">\n')
        w(_fmt(nodes.T) + "\n")
        w("        </DataArray>\n      </Points>\n")
        w("      <Cells>\n")
        w('        <DataArray type="Int64" Name="connectivity" format="ascii">\n')
        w("\n".join("         " + "".join(f" {int(v)}" for v in row) for row in (elements.T - 1)) + "\n")
        w("        </DataArray>\n")
        w('        <DataArray type="Int64" Name="offsets" format="ascii">\n')
        w("\n".join(f"          {8 * (e + 1)}" for e in range(ne)) + "\n")
        w("        </DataArray>\n")
        w('        <DataArray type="UInt8" Name="types" format="ascii">\n')
        w("\n".join("          12" for _ in range(ne)) + "\n")   # VTK_HEXAHEDRON; node order matches
        w("        </DataArray>\n      </Cells>\n")
        w('      <PointData Vectors="Displacement">\n')
        w('        <DataArray type="Float64" Name="Displacement" NumberOfComponents="3" format="ascii">\n')
        w(_fmt(Un) + "\n")
        w("        </DataArray>\n      </PointData>\n")
        w('      <CellData Scalars="VonMises" Tensors="Stress">\n')
        for name, data in (("Stress", sig_c), ("Strain", eps_c)):
            w(f'        <DataArray type="Float64" Name="{name}" NumberOfComponents="6" {comps} format="ascii">\n')
            w(_fmt(data) + "\n")
            w("        </DataArray>\n")
        for name, vals in (("VonMises", von_mises(sig_c)), ("MeanStress", sig_c[:, :3].sum(axis=1) / 3.0),
                           ("EqPlasticStrain", alp_c)):
            w(f'        <DataArray type="Float64" Name="{name}" NumberOfComponents="1" format="ascii">\n')
            w("\n".join(f"          {float(v)!r}" for v in vals) + "\n")
            w("        </DataArray>\n")
        w("      </CellData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n")
    return fn


def write_vtu(filename, model):
    """write_vtu(filename, model) (Visualization.jl:129-205) for a GPU `Model`: the
    committed Cauchy stress (finite kinds) or stress (small strain), the committed
    equivalent plastic strain and the current displacement come back through the C ABI."""
    from .model import equivalent_plastic_strain, gauss_stress
    sig = gauss_stress(model).T
    alp = equivalent_plastic_strain(model)
    return write_vtu_arrays(filename, model.mesh.nodes, model.mesh.elements, model.U, sig, alp)
