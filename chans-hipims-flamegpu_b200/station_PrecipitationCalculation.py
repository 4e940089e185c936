"""Drop-in for the reference extension module ``station_PrecipitationCalculation``
(HC/stationPrecipitation_interface.cpp:40-43)."""
from hipims_b200.ops import station_rain as addStation_Precipitation  # noqa: F401
