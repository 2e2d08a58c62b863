"""PySCF-layout molecule container and basis data (host side)."""
from .mole import Mole, M, BOHR  # noqa: F401
from .cart2sph import cart2sph_block, cart_components  # noqa: F401
