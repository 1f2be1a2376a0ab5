"""B200-native statevector engine: a drop-in for MettleQ's method="statevector" path.

Layers:
  engine.StateVector   -- kernel-level API over the C ABI (libmq.so, include/mq.h)
  device.Device        -- op-dict runtime with gate-stream fusion (reference device.py)
  integrations._common -- SDK glue (execute_operations, sampling, Pauli sums)
  adjoint              -- adjoint-method gradients, torch.autograd.Function
  batch                -- many circuits in one CUDA graph
  serving              -- continuous-batching request loop
  replicas             -- one replica per GPU for independent units
"""
from ._native import StatevectorMemoryError  # noqa: F401

__version__ = "0.1.0"


def __getattr__(name):
    if name == "StateVector":
        from .engine import StateVector
        return StateVector
    if name == "Device":
        from .device import Device
        return Device
    raise AttributeError(name)
