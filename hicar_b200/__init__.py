"""B200-native ICAR tracer-advection step (upwind / MPDATA + FCT, standard
upwind/3rd/5th order with WRF flux correction, relaxation boundaries).

The compute lives in libicar_adv.so (hand-written sm_100a CUDA behind the C
ABI of include/icar_adv.h); this package is the host-side mirror of the
reference's ``advection`` module plus the batched and served forms.
"""
from .advection import (Domain, Options, AdvOptions, PhysicsOptions, TimeOptions, Parameters, adv_init,
                        adv_var_request, advect, balance_uvw, compute_dt, mp, precipitation, restart_vars, step, step_host, kADV_MPDATA,
                        kADV_STD, kFLUXCOR_MONO, kMP_SB04)

__all__ = ["Domain", "Options", "AdvOptions", "PhysicsOptions", "TimeOptions", "Parameters", "adv_init",
           "adv_var_request", "advect", "balance_uvw", "compute_dt", "mp", "precipitation", "restart_vars", "step", "step_host",
           "kADV_MPDATA", "kADV_STD", "kFLUXCOR_MONO", "kMP_SB04"]
