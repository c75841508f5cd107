"""Geodesic-shooting surface matching under the reference's module name (reference:
base/secondOrderSurfaceMatching.py:41, imported by Examples/surfaceMatchingExample.py:20 as
`from base.secondOrderSurfaceMatching import SecondOrderSurfaceMatching`).

The class is the device-resident driver defined beside the first-order one in `base/surfaceMatching.py`; this
module only gives it the import path that unchanged reference callers use.
"""
from .surfaceMatching import SecondOrderSurfaceMatching

__all__ = ['SecondOrderSurfaceMatching']
