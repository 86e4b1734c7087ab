"""tarang_b200: B200-native pseudo-spectral IF-RK4 time stepper (FFF / SFF bases).

The compute path is the CUDA library ``libtarang_b200.so`` (hand-written
sm_100a kernels behind the C ABI in ``include/tarang_b200.h``); this package
is the host-side binding.  There is no CPU fallback.
"""
from ._lib import TsError, load as load_library, lib_path  # noqa: F401
from .adjoint import RK4Evolve, energy_norm_loss, rk4_evolve  # noqa: F401
from .solver import (Ensemble, FluidVF, Forcing, Nlin_incompress, Plan, Time_advance_incompress,  # noqa: F401
                     ensemble_members, kernel_launch_count, shard_members, spectrum_k4_gauss)

__all__ = ["Plan", "Ensemble", "RK4Evolve", "rk4_evolve", "energy_norm_loss", "ensemble_members", "shard_members", "Forcing", "FluidVF", "Nlin_incompress", "Time_advance_incompress", "TsError",
           "load_library", "lib_path", "kernel_launch_count", "spectrum_k4_gauss"]
