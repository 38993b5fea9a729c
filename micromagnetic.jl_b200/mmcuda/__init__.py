"""mmcuda -- B200 (sm_100a) finite-difference micromagnetics hot path.

Python mirror of MicroMagnetic.jl's FD API (FDMesh, Sim, set_Ms, init_m0,
add_exch, add_dmi, add_anis, add_demag, add_zeeman, run_sim, run_until,
relax, ...) on top of libmmcuda.so's C ABI (include/mmcuda.h).
"""
from ._lib import MMError, load as _load_library  # noqa: F401
from .ovf import OVF2, mag2ovf, read_ovf, save_ovf  # noqa: F401
from .adjoint import rk4_grad  # noqa: F401
from .sim import (  # noqa: F401
    FDMesh,
    Sim,
    Term,
    add_anis,
    add_demag,
    add_dmi,
    add_exch,
    add_sot,
    add_stt,
    add_thermal_noise,
    add_zeeman,
    advance_step,
    average_m,
    compute_system_energy,
    effective_field,
    init_m0,
    llg_rhs,
    mT,
    mu_0,
    relax,
    run_rk4,
    run_sim,
    run_step,
    run_until,
    set_driver,
    set_float,
    set_Ms,
    set_pinning,
    set_precision,
    update_zeeman,
    write_data,
)

__all__ = [n for n in dir() if not n.startswith("_")]
