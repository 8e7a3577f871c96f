"""cfd2d_b200: the projection time step of cfd2d on NVIDIA B200 (sm_100a).

Drop-in for the reference package's hot path: ``cases.build_case`` /
``case.sim.run``, the ``kernels`` stencil entry points and the ``pressure``
solver choice keep their names, arguments and error behaviour; the work runs in
hand-written CUDA kernels (``libcfd2d_b200.so``, C ABI in include/cfd2d_b200.h)
called through ctypes. There is no CPU fallback.
"""

from . import _lib  # noqa: F401

__version__ = "0.1.0"
__all__ = ["boundary", "cases", "geometry", "grid", "kernels", "models", "pressure", "solver",
           "turbulence", "validation"]
