"""Drop-in for the reference extension module ``fluxMask``
(HC/fluxMaskGenerator.cpp:33-35)."""
from hipims_b200.ops import flux_mask as update  # noqa: F401
