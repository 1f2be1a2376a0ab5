"""SDK adapters (Qiskit BackendV2, PennyLane device) over the B200 engine."""
