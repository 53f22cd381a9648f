"""adtlert_b200: B200 (sm_100a) forward-and-sensitivity path of AD-TLERT's 2.5D and 3D ERT operators.

Drop-in for ``adtlert.forward``'s ``ERTForward2p5D``, ``ERTForward3D`` and
``apparent_resistivity_autograd``; the
heavy work runs in ``libadtlert_b200.so`` (CUDA kernels behind a C ABI, ``include/adtlert_b200.h``).
"""

from .autograd import (
    ERT2p5DApparentResistivityFunction,
    ERT3DApparentResistivityFunction,
    ERTApparentResistivityFunction,
    apparent_resistivity_autograd,
)
from .ert2p5d import Discretization, ERTForward2p5D, ForwardResponse
from .ert3d import ERTForward3D, ForwardResponse3D
from .fem import inverse_cosine_weights, wavenumber_bounds
from .geometry import Mesh, Survey
from .geometry3d import Mesh3D
from .inputs import FLOAT_DTYPE
from .modeling import log_response_and_jacobian

__all__ = [
    "Discretization",
    "ERT2p5DApparentResistivityFunction",
    "ERT3DApparentResistivityFunction",
    "ERTApparentResistivityFunction",
    "ERTForward2p5D",
    "ERTForward3D",
    "FLOAT_DTYPE",
    "ForwardResponse",
    "ForwardResponse3D",
    "Mesh",
    "Mesh3D",
    "Survey",
    "apparent_resistivity_autograd",
    "inverse_cosine_weights",
    "log_response_and_jacobian",
    "wavenumber_bounds",
]
