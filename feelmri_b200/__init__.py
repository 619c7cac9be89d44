"""B200 (sm_100a) implementation of FEelMRI's simulation hot path.

Drop-in modules for the reference's native extensions:
  feelmri_b200.BlochSimulator.solve_mri        (feelmri.BlochSimulator)
  feelmri_b200.MRI.Signal                      (feelmri.MRI)
  feelmri_b200.Assemble.MassAssemble           (feelmri.Assemble)
  feelmri_b200.POD.tensordot_modes_weights     (feelmri.POD)
and the sequence driver feelmri_b200.Bloch.BlochSolver, which takes the
reference's BlochSolver arguments and runs a whole block sequence in one
device sweep.  Device-level entry points (torch CUDA tensors) live in
feelmri_b200.ops; the C ABI underneath is include/feelmri_b200.h
(libfeelmri_b200.so).
"""
__version__ = "0.2.0"

import importlib.abc
import sys

from . import _lib  # noqa: F401  (loads nothing until first use)

_PATCHES: dict = {}


def _apply_patch(module) -> None:
    fn = _PATCHES.get(module.__name__)
    if fn is not None:
        fn(module)


class _PatchingLoader(importlib.abc.Loader):
    def __init__(self, inner):
        self.inner = inner

    def create_module(self, spec):
        return self.inner.create_module(spec)

    def exec_module(self, module):
        self.inner.exec_module(module)
        _apply_patch(module)


class _PatchingFinder(importlib.abc.MetaPathFinder):
    """Patches reference modules (feelmri.Bloch, feelmri.Motion) right after
    they are first executed."""

    def find_spec(self, fullname, path, target=None):
        if fullname not in _PATCHES:
            return None
        for finder in sys.meta_path:
            if finder is self or not hasattr(finder, "find_spec"):
                continue
            spec = finder.find_spec(fullname, path, target)
            if spec is not None and spec.loader is not None:
                spec.loader = _PatchingLoader(spec.loader)
                return spec
        return None


_finder = _PatchingFinder()


def install_as_feelmri(device_pod: bool = False) -> None:
    """Makes the reference's Python package run on this library, unchanged.

    * feelmri.BlochSimulator, feelmri.MRI, feelmri.Assemble and feelmri.POD
      resolve to the drop-in modules here.
    * feelmri.Bloch.BlochSolver becomes feelmri_b200.Bloch.BlochSolver (same
      constructor arguments; the whole block sequence runs in one sweep).
    * With device_pod=True, feelmri.Motion.POD.calculate_pod forms the
      snapshot products on the GPU (feelmri_b200.motion.calculate_pod_on_device).

    Modules already imported are patched at once; the others when they are
    first imported."""
    from . import Assemble, BlochSimulator, MRI, POD
    from .Bloch import BlochSolver
    for name, mod in (("BlochSimulator", BlochSimulator), ("MRI", MRI), ("Assemble", Assemble), ("POD", POD)):
        sys.modules[f"feelmri.{name}"] = mod

    def patch_bloch(module):
        module.BlochSolver = BlochSolver

    _PATCHES["feelmri.Bloch"] = patch_bloch
    if device_pod:
        from .motion import calculate_pod_on_device

        def patch_motion(module):
            pod = getattr(module, "POD", None)
            if pod is not None:
                pod.calculate_pod = calculate_pod_on_device

        _PATCHES["feelmri.Motion"] = patch_motion
    for name in list(_PATCHES):
        if name in sys.modules:
            _apply_patch(sys.modules[name])
    if _finder not in sys.meta_path:
        sys.meta_path.insert(0, _finder)
