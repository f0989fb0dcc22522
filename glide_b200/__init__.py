"""glide_b200: GLIDE's SSA forward/adjoint hot path as sm_100a kernels behind the IcePhysics API.

The compute path is the native library ``libglide_b200.so`` (C ABI in
``include/glide_b200.h``); there is no CPU fallback.
"""
from .physics import (IcePhysics, abs_grad, abs_loss, huber_grad, huber_loss,  # noqa: F401
                      tikhonov_regularization)
from .grid import Grid  # noqa: F401
from .kernels import (get_kernels, make_physics_params, prolongate_cell_centered,  # noqa: F401
                      prolongate_hfacet, prolongate_vfacet, restrict_cell_centered, restrict_hfacet,
                      restrict_max_pool, restrict_vfacet)
from .solver import (SolverSettings, adjoint_vcycle, fascd_vcycle,  # noqa: F401
                     restrict_parameters_to_hierarchy)

__version__ = "0.1.0"
