"""B200 (sm_100a) implementation of FEelMRI's simulation hot path.

Drop-in modules for the reference's native extensions:
  feelmri_b200.BlochSimulator.solve_mri        (feelmri.BlochSimulator)
  feelmri_b200.MRI.Signal                      (feelmri.MRI)
  feelmri_b200.Assemble.MassAssemble           (feelmri.Assemble)
  feelmri_b200.POD.tensordot_modes_weights     (feelmri.POD)
Device-level entry points (torch CUDA tensors) live in feelmri_b200.ops; the
C ABI underneath is include/feelmri_b200.h (libfeelmri_b200.so).
"""
__version__ = "0.1.0"

from . import _lib  # noqa: F401  (loads nothing until first use)


def install_as_feelmri() -> None:
    """Registers the drop-in modules under the reference's names
    (feelmri.BlochSimulator, feelmri.MRI, feelmri.Assemble, feelmri.POD) so
    that the reference's Python package imports them unchanged."""
    import sys
    from . import Assemble, BlochSimulator, MRI, POD
    for name, mod in (("BlochSimulator", BlochSimulator), ("MRI", MRI), ("Assemble", Assemble), ("POD", POD)):
        sys.modules[f"feelmri.{name}"] = mod
