"""The shortcut of the SetupPoisson cell check (csrc/poisson.cu,
k_setup_poisson), restated in numpy and compared with the full check on
random and special doubles.

The reference's check (check_and_debug_Poisson / check_poisson_setup,
modules.f90) fails a cell when any of A1..A8 is NaN or when
A7 = A1 + .. + A6 (summed in that order) is below 1e-50.  The device forms
the west, south and bottom quotients A1, A3, A5 (which the neighbours store as
their A2, A4, A6) only when it cannot decide the check without them: when all
three quotients are numbers >= 0 by the signs of their operands, A2, A4, A6
are >= 0 and one of them is >= 1e-50, then A7 >= 1e-50 and no A is NaN
(each rounded partial sum of non-negative terms is at least its last term),
and only A8 can fail the cell."""
import math

import numpy as np
from hypothesis import given, settings, strategies as st

SPECIAL = [0.0, -0.0, 1e-300, -1e-300, 1e-60, 1e-50, 2e-50, 1.0, -1.0, 3.5, 1e300, -1e300, math.inf, -math.inf,
           math.nan, 5e-324, -5e-324]


def quot_nonneg(num, den):
    if math.isinf(num) and math.isinf(den):
        return False
    return (num >= 0.0 and den > 0.0) or (num <= 0.0 and den < 0.0)


def div(a, b):
    with np.errstate(all="ignore"):
        return float(np.float64(a) / np.float64(b))


def add(a, b):
    with np.errstate(all="ignore"):
        return float(np.float64(a) + np.float64(b))


def full_check(nums, dens, a8):
    """bad under the reference's check: NaN in A1..A8 or A7 < 1e-50."""
    a = [div(n, d) for n, d in zip(nums, dens)]
    a7 = a[0]
    for t in a[1:]:
        a7 = add(a7, t)
    return any(x != x for x in a) or a7 != a7 or a8 != a8 or a7 < 1e-50


def shortcut_check(nums, dens, a8):
    """bad as k_setup_poisson decides it."""
    a2, a4, a6 = (div(nums[q], dens[q]) for q in (1, 3, 5))
    bad = a8 != a8
    decided = (quot_nonneg(nums[0], dens[0]) and quot_nonneg(nums[2], dens[2]) and quot_nonneg(nums[4], dens[4])
               and a2 >= 0.0 and a4 >= 0.0 and a6 >= 0.0 and max(a2, a4, a6) >= 1e-50)
    if not decided:
        return full_check(nums, dens, a8)
    return bad


doubles = st.one_of(st.sampled_from(SPECIAL), st.floats(allow_nan=True, allow_infinity=True),
                    st.floats(min_value=1e-70, max_value=1e10))


@settings(max_examples=2500, deadline=None)
@given(st.lists(doubles, min_size=6, max_size=6), st.lists(doubles, min_size=6, max_size=6), doubles)
def test_shortcut_equals_full_check(nums, dens, a8):
    assert shortcut_check(nums, dens, a8) == full_check(nums, dens, a8)


def test_shortcut_on_typical_cells():
    """Coefficients of the size a 256^3 drop problem produces, and the
    wall, heavy-fluid and NaN cases of the GPU tests."""
    rng = np.random.default_rng(0)
    h = 1.0 / 256
    for _ in range(2000):
        rho = rng.choice([1.0, 1000.0], size=7) * rng.uniform(0.5, 2.0, size=7)
        nums = [2.0 * 1e-3 * m for m in rng.choice([0.0, 1.0], size=6, p=[0.1, 0.9])]
        dens = [h * h * (rho[q + 1] + rho[0]) for q in range(6)]
        for case in range(4):
            d = list(dens)
            if case == 1:
                d[rng.integers(6)] = math.nan
            elif case == 2:
                d = [x * 1e60 for x in d]
            elif case == 3:
                d[rng.integers(6)] = -d[0]
            a8 = math.nan if rng.random() < 0.05 else float(rng.standard_normal())
            assert shortcut_check(nums, d, a8) == full_check(nums, d, a8)
