"""omi_physics_b200 — the omi_physics rigid-body step on NVIDIA B200 (sm_100a).

* :class:`PhysicsWorld` — the reference's world API over the same
  structure-of-arrays columns, stepped on the GPU;
* :class:`CudaBackend` — a drop-in ``backend=`` for the reference's own
  ``omi_physics.PhysicsWorld``;
* :class:`WorldBatch` — many independent worlds stepped by the same launches;
* :class:`Server` — continuous-batching request loop under an HBM budget.

All compute runs in hand-written CUDA kernels (``csrc/``) behind the C ABI in
``include/omi_b200.h``; there is no CPU path.
"""
from . import joints, model
from ._lib import OmiError, OutOfBudget, UnsupportedFeature
from .backend import CudaBackend, select_backend
from .batch import Contact, WorldBatch
from .world import PhysicsWorld

__version__ = '0.1.0'

__all__ = ['PhysicsWorld', 'CudaBackend', 'WorldBatch', 'Contact', 'select_backend', 'model',
           'joints', 'OmiError', 'OutOfBudget', 'UnsupportedFeature', '__version__']
