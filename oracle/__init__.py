"""CPU oracle for the statevector hot path.

TEST INFRASTRUCTURE ONLY.  This package restates, in numpy, the reference's
CPU statevector algorithm (MettleQ ``sim.py`` / ``gates.py`` /
``device.py:_apply``) and the project's own seeded sampling stream.  It is the
checker that the CUDA engine is compared against.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and reference legs
may import it; the product package ``mettleq_b200`` never does.

``oracle/mlx_shim`` is a numpy-backed ``mlx.core`` stand-in under which the
reference's own CPU statevector code runs unchanged (MLX exists only for
Apple silicon): the golden generator and ``bench.py --impl reference`` use it.

Parity pin: ``tests/golden/`` holds vectors produced by running the
reference's own ``Device(n, execution_device="cpu")`` code (through that
stand-in) together with
the independent QFT matrix and affine-inverse property checks from the
reference test-suite; ``tests/test_oracle_golden.py`` checks this oracle
against them.  Sampled counts are pinned to the project's Philox4x32-10
stream (Random123 known-answer vectors), not to MLX's generator, which is
unavailable outside MLX.
"""
from .sv import (  # noqa: F401
    OracleSim,
    gate_matrix,
    compose_inverse_affine,
    qft_matrix_without_swaps,
)
from .sampler import (  # noqa: F401
    philox4x32_10,
    uniforms,
    sample_indices,
    marginal_probabilities,
    block_sums,
)
