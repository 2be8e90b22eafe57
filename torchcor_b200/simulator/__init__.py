"""Simulators (``torchcor.simulator`` names)."""
from torchcor_b200.simulator.batch import MonodomainBatch
from torchcor_b200.simulator.monodomain import Monodomain

__all__ = ["Monodomain", "MonodomainBatch"]
