"""torchcor_b200: a B200-native implementation of TorchCor's monodomain time step.

The public surface mirrors ``torchcor`` (``torchcor/__init__.py:1-4``):
``set_device``, ``get_device``, ``float32``, ``float64``; the simulator lives in
``torchcor_b200.simulator`` and the ionic models in ``torchcor_b200.ionic``.
Compute runs in hand-written sm_100a kernels of ``libtcb200.so`` (loaded on
first use by ``torchcor_b200._lib``); there is no CPU fallback.
"""
import torch

from torchcor_b200.device import get_device, set_device

float32 = torch.float32
float64 = torch.float64

__all__ = ["set_device", "get_device", "float32", "float64"]
