"""B200 engine for HFPx3D's displacement-discontinuity BEM path:
assembly -> dense LU solve -> stress, behind the C-ABI of include/hfpx_engine.h."""
from . import meshgen  # noqa: F401
