"""B200-native lattice Boltzmann sweep behind lbmpy's API.

The public names mirror lbmpy (``LBMConfig``, ``LBMOptimisation``, ``create_lb_function``,
``LatticeBoltzmannStep``, ``NoSlip``, ``UBB``, the macroscopic getter/setter, the scenarios);
the sweep itself is hand-written CUDA for sm_100a in ``liblbmb200.so`` (C ABI:
``include/lbm_b200.h``), reached through ctypes with PyTorch tensors owning the fields.
"""
from .enums import (CollisionSpace, ForceModel, Method, Stencil, SubgridScaleModel, Target, Timestep,  # noqa: F401
                    get_timesteps, is_inplace)
from .stencils import LBStencil  # noqa: F401
from .creationfunctions import (CreateKernelConfig, LBMConfig, LBMOptimisation, create_lb_ast,  # noqa: F401
                                create_lb_collision_rule, create_lb_function, create_lb_method,
                                create_lb_update_rule, update_with_default_parameters)
from .relaxationrates import (lattice_viscosity_from_relaxation_rate,  # noqa: F401
                              relaxation_rate_from_lattice_viscosity, relaxation_rate_from_magic_number)
from .fields import create_pdf_array  # noqa: F401
from .boundaries import (NoSlip, UBB, FixedDensity, FreeSlip, SimpleExtrapolationOutflow,  # noqa: F401
                         ExtrapolationOutflow, NoSlipLinearBouzidi, LatticeBoltzmannBoundaryHandling,
                         slice_from_direction)
from . import geometry  # noqa: F401
from .macroscopic_value_kernels import (compile_macroscopic_values_getter,  # noqa: F401
                                        compile_macroscopic_values_setter, macroscopic_values_getter,
                                        macroscopic_values_setter, pdf_initialization_assignments)
from .lbstep import LatticeBoltzmannStep  # noqa: F401
from .scenarios import create_channel, create_fully_periodic_flow, create_lid_driven_cavity  # noqa: F401
