"""Counterpart of ``byteqc.cuobc``: the GPU J/K path."""
from byteqc_b200.cuobc import scf  # noqa: F401
