"""Drop-in for the reference extension module
``fluxCalculation_jh_modified_surface`` (HC/fluxCal_jh_modified_surface.cpp:55-57):
``addFlux`` runs the B200 1st-order (bed-only minmod) HLLC flux op."""
from hipims_b200.ops import flux_1st_order as addFlux  # noqa: F401
