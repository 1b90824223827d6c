"""B200-native engine for pyGCMC's hot path: fragment-environment LJ+Coulomb
trial-move energies with cavity-bias insertion and on-device accept/update.

Drop-in entry: :func:`pygcmc_b200.gpu.runGCMC` (same call as ``gcmc.gpu.runGCMC``).
"""
from . import values  # noqa: F401

__all__ = ["values", "gpu", "engine", "system"]
