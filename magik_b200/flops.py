"""Algorithmic operation counts of the integrator, used for the roofline.

The roofline counts the work of the reference's algorithm, not of this
library's formulation: source-level counts (+, -, *, /, sqrt = 1; a fused
multiply-add = 2) of the reference's expression trees for the RHS
(metric_kerr.cuh:38-105, metric_schwarzschild.cuh:8-72) and the RKF45
attempt (internal_math.h:2160-2205, relativity_utilities.cuh:10-55) on its
8-component state.  The CPU oracle evaluates those trees with an
op-counting scalar; tests/test_host.py checks the figures below against it.

  RHS            Kerr 156          Schwarzschild 126
  RKF45 attempt  Kerr 1398         Schwarzschild 1218  (6 RHS + stage
                 combinations, 5th-order solution, error, norm, proposal)

A crossing sub-step (the secant refinement of a disk or escape crossing, an
addition of this library) is counted as 6 RHS of the reference tree plus
its 300 stage-combination operations.

The kernels execute fewer operations than that (the fused RHS of the MIXED
and F64 modes, and 7 state components: dp_t/dl = 0 is not integrated);
IMPLEMENTATION holds those counts (RHS, attempt) for information.
"""

RHS = {2: 156, 1: 126, 0: 0}
ATTEMPT = {2: 1398, 1: 1218, 0: 0}
SUBSTEP_OVERHEAD = 300

# operations of the fused formulation the MIXED / F64 kernels run, counted by
# the oracle on its 8-component state: (RHS, attempt)
IMPLEMENTATION = {2: (105, 1092), 1: (38, 690)}


def attempt_flops(metric):
    return ATTEMPT[metric]


def substep_flops(metric):
    return 6 * RHS[metric] + SUBSTEP_OVERHEAD


def render_flops(metric, attempts, refine_evals):
    return attempts * attempt_flops(metric) + refine_evals * substep_flops(metric)
