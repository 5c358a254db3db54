"""B200 (sm_100a) implementation of NeuralPOM's physical time step.

The explicit mode-split and semi-implicit free-surface POM cores advance on
the GPU through ``libnpom_b200.so`` (C ABI in ``include/npom.h``); this
package holds the host side: the drop-in core classes, the physics executor
and the case builders.
"""
from . import _abi, cases, state  # noqa: F401
from .core import B200Core, ExplicitCore, ImplicitCore, CORE_REGISTRY, resolve_core_class  # noqa: F401
from .physics import B200Physics  # noqa: F401

__all__ = ["B200Core", "ExplicitCore", "ImplicitCore", "B200Physics", "CORE_REGISTRY", "resolve_core_class",
           "load_library"]


def load_library():
    return _abi.load_library()
