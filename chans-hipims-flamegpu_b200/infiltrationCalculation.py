"""Drop-in for the reference extension module ``infiltrationCalculation``
(HC/infiltration_interface.cpp): Green-Ampt infiltration."""
from hipims_b200.ops import infiltration as addinfiltration  # noqa: F401
