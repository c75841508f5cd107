"""CPU oracle for the py-lddmm point-set hot path -- TEST INFRASTRUCTURE ONLY.

This package is a float64 CPU restatement of the reference algorithms (numba `prange` loops, the same CPU
technology as the reference's `_numba` kernels). It exists to check the CUDA path and to time a CPU
baseline. Only `tests/`, `__graft_entry__.smoke()` and `bench.py` (its `cpu_baseline` leg and its
`--impl reference` arm) may import it, and only as the checker or the timed CPU baseline -- never as the
product path. The package `py-lddmm_b200/` never imports it.

Parity pinning: every function here is checked against golden fixtures produced by running the
reference itself (tests/golden/make_golden.py, tests/test_oracle_golden.py).
"""
from .kernels import (apply_k, apply_diff_kt, apply_ddiff_k11and12, apply_diff_k1and2, apply_divergence,
                      apply_k_tensor, apply_k_mat, apply_diff_k_mat)
from . import laplacian
from .shooting import (landmark_direct_evolution_euler, landmark_hamiltonian_gradient, landmark_epdiff,
                       second_order_evolution, second_order_gradient, second_order_step_rows,
                       second_order_adjoint_step_rows)
from .surface_terms import (face_geometry, varifold_norm0, varifold_norm_def, varifold_norm_gradient,
                            varifold_norm_gradient_rows,
                            current_norm0, current_norm_def, current_norm_gradient,
                            measure_norm0, measure_norm_def, measure_norm_gradient)
