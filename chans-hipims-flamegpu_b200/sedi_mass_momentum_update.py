"""Import-only stand-in for the reference extension module ``sedi_mass_momentum_update``.

The reference solver imports it at module load (HP/SWE_CUDA.py:29-41); its op
is outside the B200 hot path, so calling it raises NotImplementedError."""


def add_source(*args, **kwargs):
    raise NotImplementedError("sedi_mass_momentum_update.add_source is not part of the B200 HiPIMS step")
