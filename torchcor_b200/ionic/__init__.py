"""Ionic models (``torchcor.ionic`` names)."""
from torchcor_b200.ionic.models import (CourtemancheRamirezNattel, MitchellSchaeffer, ModifiedMS2v,
                                        TenTusscherPanfilov)

__all__ = ["ModifiedMS2v", "MitchellSchaeffer", "TenTusscherPanfilov", "CourtemancheRamirezNattel"]
