"""Counterpart of ``byteqc.cuobc.scf`` (cuobc/scf/__init__.py:34-35)."""
from byteqc_b200.cuobc.scf import hf  # noqa: F401
from byteqc_b200.cuobc.scf.hf import get_jk, _VHFOpt, RHF  # noqa: F401
