"""Drop-in for the reference extension module ``euler_update``
(HC/euler_update.cpp:46-48)."""
from hipims_b200.ops import euler_update as update  # noqa: F401
