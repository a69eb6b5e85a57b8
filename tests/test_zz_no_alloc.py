"""pfem_norm2_noalloc: the residual norm computed without any device allocation.

Callers that cannot allocate device memory (their framework owns every device
allocation, or their steady state must not call cudaMalloc/cudaFree) pass the
vector and a one-element result buffer they already own.  This file runs last
so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import _lib as L
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _residual_case():
    w = W.config0(n=6, nsteps=4)
    M = P.Model(w.mesh, P.J2Material(**w.material))
    w.apply(M)
    X = w.mesh.nodes
    U = np.stack([0.002 * X[0], -0.001 * X[1], 0.004 * X[2]]).T.reshape(-1)
    U += 1e-4 * np.sin(np.arange(U.size))
    M.set_displacement(U)
    rnorm, R = M.residual(0.5)          # existing entry point: norm via allocated scratch
    return M, rnorm, R


def test_norm2_noalloc_matches_residual_norm():
    import torch
    M, rnorm, R = _residual_case()
    assert rnorm > 0
    x = torch.tensor(R, dtype=torch.float64, device="cuda:0")
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    lib = L.lib()
    for _ in range(2):                   # two calls in a row share the scratch array
        out.zero_()
        rc = lib.pfem_norm2_noalloc(C.c_void_p(x.data_ptr()), x.numel(), C.c_void_p(out.data_ptr()),
                                    C.c_void_p(stream))
        assert rc == L.PFEM_OK, lib.pfem_last_error(None)
        torch.cuda.synchronize(0)
        assert abs(out.item() - rnorm) <= 1e-12 * rnorm
    # a smaller vector after a larger one: stale partial sums must not leak in
    y = x[:1000].clone()
    rc = lib.pfem_norm2_noalloc(C.c_void_p(y.data_ptr()), y.numel(), C.c_void_p(out.data_ptr()),
                                C.c_void_p(stream))
    assert rc == L.PFEM_OK
    torch.cuda.synchronize(0)
    ref = float(np.linalg.norm(R[:1000]))
    assert abs(out.item() - ref) <= 1e-12 * ref


def test_norm2_noalloc_rejects_oversize():
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    x = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    lib = L.lib()
    rc = lib.pfem_norm2_noalloc(C.c_void_p(x.data_ptr()), 134_217_728 + 1, C.c_void_p(out.data_ptr()), None)
    assert rc == L.PFEM_ERR_BAD_ARG
    assert b"exceeds the maximum" in lib.pfem_last_error(None)
