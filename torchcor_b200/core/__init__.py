"""Mesh input, conductivities, stimuli and device assembly (``torchcor.core`` names)."""
from torchcor_b200.core.assemble import Matrices3D, Matrices3DSurface, assemble_system, build_pattern
from torchcor_b200.core.conductivity import Conductivity
from torchcor_b200.core.mesh import MeshReader, read_vtx
from torchcor_b200.core.stimulation import StimConfig, Stimuli

__all__ = ["MeshReader", "read_vtx", "Conductivity", "Stimuli", "StimConfig", "Matrices3D", "Matrices3DSurface",
           "assemble_system", "build_pattern"]
