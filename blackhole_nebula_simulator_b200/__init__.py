"""B200-native SPH step of Blackhole-Nebula-Simulator.

Drop-in modules with the reference's names: ``coupled`` (shared step), ``blocks`` (block time
steps), ``ops`` (find_neighbours, tighten, density_numba, forces_numba, disc_forces_numba,
glf_step_many, gn_v_from_p, beta_cool), ``cooling`` (bremsstrahlung), ``config`` (HydroConfig,
CoupledConfig, BlockConfig).  The arithmetic runs in libnebula_b200.so (hand-written sm_100a
CUDA behind the C ABI of include/nebula_b200.h); PyTorch only holds device memory and streams.
"""

from . import config, ics, units  # noqa: F401

__all__ = ["config", "ics", "units", "ops", "coupled", "blocks", "cooling", "build"]
