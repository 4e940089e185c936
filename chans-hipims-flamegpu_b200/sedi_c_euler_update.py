"""Import-only stand-in for the reference extension module ``sedi_c_euler_update``.

The reference solver imports it at module load (HP/SWE_CUDA.py:29-41); its op
is outside the B200 hot path, so calling it raises NotImplementedError."""


def update(*args, **kwargs):
    raise NotImplementedError("sedi_c_euler_update.update is not part of the B200 HiPIMS step")
