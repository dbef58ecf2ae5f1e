"""B200 element loop of sparlab_form: incompatible-mode Hex8 elements with
logarithmic-strain kinematics and the J2 / Hill48 return map under
isotropic, Prager and Chaboche hardening, their local Newton iteration and
static condensation, the assembly into the node-block pattern and penalty
contact with rigid tools, and the free-free tangent of a Dirichlet
partition fed to a device sparse factorisation, and the release step's
adjoint with respect to the reference geometry - hand-written CUDA for
sm_100a in libsbk.so (include/sbk.h), wrapped here behind the reference's
own interfaces.
"""
from . import _capi
from ._capi import SbkError, SolverError
from .adjoint import BicubicHeights, Release, ReleaseFunction, compensate, released, springback_rms, supports_321
from .contact import ToolContact, Tool
from .material import Material
from .mesh import HexMesh, structured_hex_mesh
from .partition import PartitionedFactor
from .system import Evaluation, NonlinearSystem, element_batch

__all__ = ["Material", "HexMesh", "structured_hex_mesh", "NonlinearSystem", "Evaluation", "element_batch",
           "ToolContact", "Tool", "SbkError", "SolverError", "PartitionedFactor",
           "BicubicHeights", "Release", "ReleaseFunction", "compensate", "released", "springback_rms",
           "supports_321"]


def library_path() -> str:
    return _capi.LIB_PATH
