"""CPU tests of the product's host-side topology and its C ABI (no GPU needed).

The sparsity pattern and colors must match the reference bit-exactly
(Assembly.jl:99-206, pinned by test_assembly.jl:26-35); the oracle restates
that algorithm, so both are compared here.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import _lib as L
from plasticity_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAT = P.J2Material(210e3, 0.3, 250.0, 1000.0)


def test_library_exports_every_header_symbol():
    hdr = open(os.path.join(ROOT, "include", "pfem_b200.h")).read()
    names = set(re.findall(r"^\s*(?:int64_t|int|void|const char\*)\s+(pfem_\w+)\s*\(", hdr, re.M))
    assert len(names) >= 17
    lib = L.lib()
    for n in names:
        assert hasattr(lib, n), n
    assert names == set(L.SIGNATURES), names ^ set(L.SIGNATURES)


def test_bad_arguments_rejected():
    lib = L.lib()
    ctx = C.c_void_p()
    nodes = np.zeros((8, 3)); el = np.arange(1, 9, dtype=np.int64).reshape(1, 8)
    # test_saturation.jl:128-140 (T15): saturation with Hkin > 0, sigsat < sigy0, delta < 0
    for m in (L.Material(206.9e3, 0.29, 450.0, 129.24, 100.0, 715.0, 16.93),
              L.Material(210e3, 0.3, 450.0, 0.0, 0.0, 400.0, 10.0),
              L.Material(210e3, 0.3, 450.0, 0.0, 0.0, 715.0, -1.0)):
        rc = lib.pfem_create(C.byref(ctx), L.ptr(nodes), 8, L.ptr(el, L._i64), 1, 2, C.byref(m), None, -1)
        assert rc == L.PFEM_ERR_BAD_ARG
    for kw in (dict(sigsat=715.0, delta=16.93, Hiso=129.24, Hkin=100.0), dict(sigsat=400.0, delta=10.0),
               dict(sigsat=715.0, delta=-1.0)):
        with pytest.raises(ValueError):
            P.J2Material(210e3, 0.3, 450.0, **kw)
    mlin = P.J2Material(210e3, 0.3, 250.0, Hiso=1000.0)
    assert mlin.sigsat == mlin.sigy0 and mlin.delta == 0.0
    # kinematic and saturation materials are accepted (topology-only context)
    for m in (L.Material(210e3, 0.3, 250.0, 200.0, 2000.0, 0.0, 0.0),
              L.Material(206.9e3, 0.29, 450.0, 129.24, 0.0, 715.0, 16.93)):
        c2 = C.c_void_p()
        rc = lib.pfem_create(C.byref(c2), L.ptr(nodes), 8, L.ptr(el, L._i64), 1, 2, C.byref(m), None, -1)
        assert rc == 0
        lib.pfem_destroy(c2)
    m = L.Material(210e3, 0.6, 250.0, 0.0, 0.0)            # nu >= 0.5 (Materials.jl:91)
    rc = lib.pfem_create(C.byref(ctx), L.ptr(nodes), 8, L.ptr(el, L._i64), 1, 2, C.byref(m), None, -1)
    assert rc == L.PFEM_ERR_BAD_ARG
    el[0, 0] = 99                                           # node id out of range
    m = L.Material(210e3, 0.3, 250.0, 0.0, 0.0)
    rc = lib.pfem_create(C.byref(ctx), L.ptr(nodes), 8, L.ptr(el, L._i64), 1, 2, C.byref(m), None, -1)
    assert rc == L.PFEM_ERR_BAD_ARG
    with pytest.raises(ValueError):
        P.J2Material(210e3, 0.5, 250.0)


def test_topology_only_context_refuses_compute():
    M = P.Model(P.box_mesh(1, 1, 1, 1, 1, 1), MAT, device=-1)
    with pytest.raises(P.PfemError) as e:
        M.assemble(np.zeros(M.ndof))
    assert e.value.code == L.PFEM_ERR_STATE


@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 2, 4), (5, 1, 1), (4, 4, 4)])
def test_pattern_bit_exact_vs_oracle(oracle, dims):
    mesh = P.box_mesh(1.0, 2.0, 1.5, *dims)
    M = P.Model(mesh, MAT, device=-1)
    cp, rv = M.pattern()
    ocp, orv = oracle.pattern(mesh.nnodes, mesh.elements)
    assert cp.dtype == np.int64 and np.array_equal(cp, ocp) and np.array_equal(rv, orv)


def test_pattern_jittered_mesh_and_colors(oracle):
    w = W.config2(n=6)
    M = P.Model(w.mesh, MAT, device=-1)
    cp, rv = M.pattern()
    ocp, orv = oracle.pattern(w.mesh.nnodes, w.mesh.elements)
    assert np.array_equal(cp, ocp) and np.array_equal(rv, orv)
    # perturbed coordinates: the reference's coordinate-based colors collapse to 1 (Assembly.jl:175-177)
    nc, col = M.colors()
    onc, ocol = oracle.element_colors(w.mesh.nodes, w.mesh.elements)
    assert nc == onc == 1 and np.array_equal(col, ocol)


@pytest.mark.parametrize("dims", [(2, 2, 2), (3, 3, 1), (1, 1, 1), (4, 3, 2)])
def test_colors_bit_exact_vs_oracle(oracle, dims):
    mesh = P.box_mesh(1, 1, 1, *dims)
    M = P.Model(mesh, MAT, device=-1)
    nc, col = M.colors()
    onc, ocol = oracle.element_colors(mesh.nodes, mesh.elements)
    assert nc == onc and np.array_equal(col, ocol)
    # same-color elements share no node
    el = mesh.elements
    for c in range(nc):
        ids = np.nonzero(col == c)[0]
        nodes = el[:, ids].ravel()
        assert len(np.unique(nodes)) == len(nodes)


def test_mesh_helpers_match_oracle(oracle):
    m = P.box_mesh(2.0, 1.0, 3.0, 3, 2, 4)
    on, oe = oracle.box_mesh(2.0, 1.0, 3.0, 3, 2, 4)
    assert np.array_equal(m.nodes, on) and np.array_equal(m.elements, oe)
    assert list(P.on_face(m, "xmax")) == [i + 1 for i in range(m.nnodes) if abs(m.nodes[0, i] - 2.0) <= 1e-8 * 3]
    assert list(P.dof(np.array([1, 2]), 3)) == [3, 6]


def test_workload_shapes():
    w = W.config2(n=8)
    assert w.mesh.nelem == 512 and w.sigy0_e.shape == (512,)
    assert abs(w.sigy0_e.mean() / 250 - 1) < 0.05
    X = w.mesh.nodes
    assert X.min() == 0 and X.max() == 1.0
    w0 = W.config0()
    assert w0.mesh.nnodes == 729 and 3 * w0.mesh.nnodes == 2187
    w1 = W.config1(nx=8, ny=2, nz=2)
    assert (w1.sigy0_e < 250).sum() == 4
    w3 = W.config3(n=12, patch=4)
    assert (w3.dir_vals < 0).sum() == 16


def test_boundary_condition_changes_mark_model_dirty():
    """Re-applying a different load path's BCs to a reused model must be pushed
    to the device before the next solve."""
    w1 = W.config4_path(n=3, seed=1)
    w2 = W.config4_path(n=3, seed=2)
    M = P.Model(w1.mesh, P.J2Material(**w1.material), device=-1)
    w1.apply(M)
    assert M._bcs_dirty
    M._bcs_dirty = False          # as after a push
    w2.apply(M)
    assert M._bcs_dirty
    assert not np.allclose(w1.dir_vals, w2.dir_vals)
    M._bcs_dirty = False
    M.prescribe([1], "x", 0.1)
    assert M._bcs_dirty


def test_bc_builders_match_oracle_loops(oracle):
    """fix!/prescribe!/load! (Model.jl:102-145): the vectorised builders give the
    oracle's node-major dof order, values and ramp flags; after Workload.apply
    (arrays) further builder calls extend the arrays."""
    mesh = P.box_mesh(1.0, 2.0, 1.0, 3, 2, 2)
    M = P.Model(mesh, MAT, device=-1)
    om = oracle.OracleModel(mesh.nodes, mesh.elements, oracle.J2Material(210e3, 0.3, 250.0, 1000.0))
    for m in (M, om):
        m.fix(P.on_face(mesh, "zmin"), "all")
        m.fix(P.on_face(mesh, "xmin"), "x")
        m.prescribe(P.on_face(mesh, "xmax"), "y", -0.02)
        m.prescribe(P.on_face(mesh, "zmax"), "z", 0.01, ramp=False)
        m.load(P.on_face(mesh, "ymax"), "x", 6.0, distribute=True)
    assert np.array_equal(np.asarray(M.dir_dofs), np.asarray(om.dir_dofs))
    assert np.array_equal(np.asarray(M.dir_vals), np.asarray(om.dir_vals))
    assert np.array_equal(np.asarray(M.dir_ramp, bool), np.asarray(om.dir_ramp, bool))
    assert np.array_equal(np.asarray(M.neu_dofs), np.asarray(om.neu_dofs))
    assert np.allclose(np.asarray(M.neu_vals), np.asarray(om.neu_vals), rtol=0, atol=0)
    w = W.config2(n=3)
    w.apply(M)
    n0 = len(M.dir_dofs)
    M.fix([1], "z")
    assert len(M.dir_dofs) == n0 + 1 and M.dir_dofs[-1] == 3 and M._bcs_dirty


def test_abi_structs_match_header():
    """The ctypes mirrors of pfem_material, pfem_solve_opts and pfem_solve_result
    list the header's fields in order with the same C types (the library writes
    through these structs, so a mismatch would corrupt memory)."""
    hdr = open(os.path.join(ROOT, "include", "pfem_b200.h")).read()
    ctype = {"int32_t": C.c_int32, "double": C.c_double, "int64_t": C.c_int64}
    for cname, pycls in (("pfem_material", L.Material), ("pfem_solve_opts", L.SolveOpts),
                         ("pfem_solve_result", L.SolveResultC)):
        body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (cname, cname), hdr, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            t, names = decl.split(None, 1)
            fields += [(n.strip(), ctype[t]) for n in names.split(",")]
        assert [(n, t) for n, t in pycls._fields_] == fields, cname
