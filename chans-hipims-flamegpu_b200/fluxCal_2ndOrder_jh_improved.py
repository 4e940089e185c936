"""Drop-in for the reference extension module ``fluxCal_2ndOrder_jh_improved``
(HC/fluxCal_2ndOrder_jh_improved.cpp:55-57): ``addFlux`` runs the B200
2nd-order MUSCL / hydrostatic / HLLC flux op of libhipims_b200."""
from hipims_b200.ops import flux_2nd_order as addFlux  # noqa: F401
