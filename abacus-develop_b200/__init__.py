"""B200-native plane-wave Kohn-Sham H|psi> and block-Davidson path of ABACUS.

Host code (C++) and hand-written sm_100a kernels live in ``csrc/`` and are
built into ``libabacus_b200.so``; this package is the Python face of that
library's C-ABI (``include/abacus_b200.h``).
"""
from . import _lib, hsolver, kpool, nscf, nscf_io, pwdft, serve, synth  # noqa: F401

__all__ = ["synth", "_lib", "pwdft", "kpool", "serve", "nscf_io", "nscf", "hsolver"]
