"""B200-native (sm_100a) residual-and-update path of the aerocfd multi-block
structured compressible-flow solver, behind a C-ABI that mirrors the
reference's Fortran subroutine interfaces."""
from .case import Block, Case, Config, Subface  # noqa: F401
