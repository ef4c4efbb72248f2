"""librint_b200: B200-native Rys-quadrature ERIs and RHF Fock builds behind
librint's C ABI.  The compute runs in the CUDA library librint_b200/_lib/
librint_b200.so (built by ``librint_b200.build``); importing a module that
needs it raises if it is missing -- there is no CPU fallback."""
from .basis import Molecule, read_molecule  # noqa: F401

__all__ = ["Molecule", "read_molecule"]
