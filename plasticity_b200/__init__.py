"""plasticity_b200 -- B200-native finite-strain F-bar J2 plasticity path.

Drop-in for the per-Newton-iteration path of vinaysrao1/plasticity's
``lagrangian/`` solver: the API mirrors ``PlasticityFEM`` (PlasticityFEM.jl:35-47)
and every numerical call runs in the CUDA library ``libpfem_b200.so`` through
its C ABI (include/pfem_b200.h).
"""
from .model import (Mesh, J2Material, Model, SolveResult, box_mesh, on_face, select_nodes, dof,
                    fix, prescribe, load, solve, reset, nodal_displacements, gauss_stress,
                    gauss_kirchhoff, equivalent_plastic_strain)
from ._lib import PfemError, lib

__all__ = ["Mesh", "J2Material", "Model", "SolveResult", "box_mesh", "on_face", "select_nodes", "dof",
           "fix", "prescribe", "load", "solve", "reset", "nodal_displacements", "gauss_stress",
           "gauss_kirchhoff", "equivalent_plastic_strain", "PfemError", "lib"]
