"""B200 implementation of BG_Flood's explicit shallow-water flow step on the
block-uniform quadtree, behind a C ABI (include/bg_flood_b200.h).

Modules:
  params  -- Param mirror and BG_param.txt key reader (reference src/Param.h, src/ReadInput.cu)
  mesh    -- BUQ mesh, halo fill and boundary-segment helpers (src/Mesh.cu, src/Halo.cu)
  flow    -- FlowB200: one scenario on one GPU (stands in for FlowGPU, src/FlowGPU.cu)
  build   -- in-tree build of the sm_100a library
"""
from .params import Param, read_param_text, BndSegmentSpec  # noqa: F401


def __getattr__(name):
    # the native pieces load lazily so that importing the package never needs a GPU
    if name in ("FlowB200", "BGFError", "Loop", "build_model"):
        from . import flow
        return getattr(flow, name)
    if name in ("Mesh", "uniform_mesh", "grid_to_buq", "buq_to_grid", "fill_halo", "boundary_segments"):
        from . import mesh
        return getattr(mesh, name)
    raise AttributeError(name)
