from byteqc_b200.gto.mole import Mole, M  # noqa: F401
from byteqc_b200.gto import basis, geom  # noqa: F401
