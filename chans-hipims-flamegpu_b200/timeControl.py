"""Drop-in for the reference extension module ``timeControl``
(HC/timeControl.cpp:43-45)."""
from hipims_b200.ops import update_timestep as updateTimestep  # noqa: F401
