"""Import-only stand-in for the reference extension module ``frictionCalculation``.

The reference solver imports it at module load (HP/SWE_CUDA.py:29-41); its op
is outside the B200 hot path, so calling it raises NotImplementedError."""


def addFriction(*args, **kwargs):
    raise NotImplementedError("frictionCalculation.addFriction is not part of the B200 HiPIMS step")
