"""Drop-in for the reference extension module ``friction_implicit_andUpdate_jh``
(HC/friction_implicit_andUpdate_jh_interface.cpp:53-56)."""
from hipims_b200.ops import friction_update as addFriction_eulerUpdate  # noqa: F401
