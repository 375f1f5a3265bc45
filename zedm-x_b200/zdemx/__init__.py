"""zdemx -- the ZDEM-X polyhedral contact step on B200.

The compute runs in libzdemx.so (hand-written sm_100a CUDA behind the C ABI of include/zdemx.h);
this package is the host-side mirror of the reference's Python surface:

* ``zdemx.polyline``  -- drop-in for the reference's polyline.py (pair contacts, VTK writers, CLI).
* ``zdemx.contact``   -- the batched pair call (many pairs of meshes in one call).
* ``zdemx.synth``     -- seeded synthetic meshes and poses for the benchmarks and tests.
"""
from ._lib import Context, ZdxError, mesh_build, stl_load  # noqa: F401

__version__ = "0.1.0"
