"""B200-native SPH + Barnes-Hut particle step with the call surface of the
SPH_3 reference (``sph_code/libsx.py``, ``sph_code/shear.py``).

* :mod:`sph_3_b200.libsx`, :mod:`sph_3_b200.shear` -- the reference's
  function names and signatures, computed on the GPU.
* :class:`sph_3_b200.Context` -- a device-resident particle set (or a batch
  of systems) with the fused, CUDA-graph-captured KDK step.
* ``include/sph3.h`` -- the C ABI underneath both.
"""
from .context import Config, Context, FIELDS, STATUS_BITS  # noqa: F401
from ._lib import LibraryError, Sph3Error, load  # noqa: F401

__all__ = ["Config", "Context", "FIELDS", "STATUS_BITS", "LibraryError", "Sph3Error", "load"]
