"""Algorithmic operation counts of the integrator, used for the roofline.

Source-level counts (+, -, *, /, sqrt = 1; fused multiply-add = 2; pow = 1)
of the formulation the kernels execute (a division or a square root counts
as one operation however it is implemented): the 7-component state (x, y, z, t,
px, py, pz) with the conserved p_t carried beside it.  The CPU oracle counts
the same expressions with an op-counting scalar (8 components, p_t included);
tests/test_host.py checks that the figures below equal its counts minus the
p_t work, which is identically zero and skipped by the kernels.

  RHS                           Kerr 162   Schwarzschild 132 (the fused
                                formulation: one reciprocal and eight
                                products in place of five quotients)
  one RKF45 attempt             6 RHS + 25 coefficient products + 210 stage
                                combinations + 70 (5th-order solution)
                                + 63 (error) + 36 (norm) + 4 (proposal)
  one crossing sub-step         6 RHS + 20 coefficient products + 210 + 70
"""

RHS = {2: 162, 1: 132, 0: 0}
ATTEMPT_OVERHEAD = 25 + 210 + 70 + 63 + 36 + 4
SUBSTEP_OVERHEAD = 20 + 210 + 70
# p_t terms the 8-component count includes and the kernels skip
PT_TERMS_PER_ATTEMPT = 54


def attempt_flops(metric):
    return 6 * RHS[metric] + ATTEMPT_OVERHEAD


def substep_flops(metric):
    return 6 * RHS[metric] + SUBSTEP_OVERHEAD


def render_flops(metric, attempts, refine_evals):
    return attempts * attempt_flops(metric) + refine_evals * substep_flops(metric)
