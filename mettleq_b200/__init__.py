"""B200-native statevector engine: a drop-in for MettleQ's method="statevector" path.

Layers (see DESIGN.md at the repository root for the full map):
  engine.StateVector   -- kernel-level API over the C ABI (libmq.so)
  device.Device        -- op-dict runtime with gate-stream fusion (device.py)
  integrations._common -- SDK glue (execute_operations, sampling, Pauli sums)
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
