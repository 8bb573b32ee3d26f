"""accelerint_b200: batched stiff-ODE integration on one B200 behind accelerInt's C interface.

The product is the C-ABI shared library ``libaccelerint_b200.so`` (declared in
include/accelerint_b200.h).  This package is its Python host-side mirror: the
same three calls as the reference's library interface
(generic/solver_interface.cuh:35-55) plus the extension calls, with numpy
arrays in the reference's column-major layout ``y[i, ivp]`` (``y_host[i*NUM +
ivp]``).  There is no CPU fallback: if the library is missing, importing
``Integrator`` works but constructing one raises.
"""
from .mechanism import (MassAction, VanDerPol, mechanism_13, mechanism_53,  # noqa: F401
                        mass_action_initial_conditions, mixed_stiffness_initial_conditions,
                        synthetic_mechanism, vdp_initial_conditions)
from ._lib import (ACCELERINT_ERR_SYSTEMS, ACCELERINT_OK, EXPORTED_SYMBOLS, LU_FP32, LU_FP32_ALL, LU_FP64,  # noqa: F401
                   NSTATS, SOLVERS, Integrator, library_path, load_library)
