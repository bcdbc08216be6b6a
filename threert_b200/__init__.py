"""threert_b200: ThreeRT's offline path-trace pass (software traversal) as a wavefront of sm_100a CUDA kernels.

- `prep`: scene descriptions and the host prep that packs them into the reference's buffers;
- `gpu`: the pass (`Gpu.render`, the counterpart of renderer/src/gpu.rs `Gpu::render`) over the C ABI of
  include/threert_cuda.h;
- `scenes`: seeded synthetic scenes (Cornell box, procedural city, the analytic render tests).
"""
from .gpu import Frame, Gpu, RenderError, Scene, frame_of  # noqa: F401
from .prep import (Camera, DirLight, Instance, Material, Mesh, Prepared, Preset, SceneDescription, Sky,  # noqa: F401
                   lambert, prepare)
