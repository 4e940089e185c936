"""Import-only stand-in for the reference extension module ``fluxCalculation_convectionTranport``.

The reference solver imports it at module load (HP/SWE_CUDA.py:29-41); its op
is outside the B200 hot path, so calling it raises NotImplementedError."""


def addFlux(*args, **kwargs):
    raise NotImplementedError("fluxCalculation_convectionTranport.addFlux is not part of the B200 HiPIMS step")
