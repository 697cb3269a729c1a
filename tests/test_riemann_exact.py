"""The exact Riemann solution used to measure the batched strips' error
(finite-volume-2d-cpp_b200/riemann.py) against the star states published
with Toro's test problems (Riemann Solvers and Numerical Methods for Fluid
Dynamics, table 4.3) and the Sod solution."""
import numpy as np
import pytest

import riemann


@pytest.mark.parametrize("left,right,p_star,u_star", [
    ((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 0.30313, 0.92745),          # Sod (Toro test 1)
    ((1.0, -2.0, 0.4), (1.0, 2.0, 0.4), 0.00189, 0.0),               # test 2: two rarefactions
    ((1.0, 0.0, 1000.0), (1.0, 0.0, 0.01), 460.894, 19.5975),         # test 3
    ((1.0, 0.0, 0.01), (1.0, 0.0, 100.0), 46.0950, -6.19633),         # test 4
    ((5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950), 1691.64, 8.68975),  # test 5
])
def test_star_states(left, right, p_star, u_star):
    p, u = riemann.star_state(left, right)
    assert abs(p - p_star) <= 5e-5 * max(1.0, p_star) + 5e-6
    assert abs(u - u_star) <= 5e-5 * max(1.0, abs(u_star)) + 5e-6


def test_sod_profile_and_mirror_symmetry():
    x = np.linspace(0.0, 1.0, 2001)
    r, u, p = riemann.sample(x, 0.2, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    assert r[0] == 1.0 and r[-1] == 0.125 and p[0] == 1.0 and p[-1] == 0.1
    plateau = (x > 0.70) & (x < 0.84)      # between contact (0.6855) and shock (0.8504)
    assert np.allclose(r[plateau], 0.26557, atol=1e-5) and np.allclose(p[plateau], 0.30313, atol=1e-5)
    a = riemann.sample(x, 0.1, (0.3, 0.2, 0.5), (0.8, -0.4, 0.2))
    b = riemann.sample(1.0 - x, 0.1, (0.8, 0.4, 0.2), (0.3, -0.2, 0.5))
    assert np.allclose(a[0], b[0]) and np.allclose(a[1], -b[1]) and np.allclose(a[2], b[2])


def test_vacuum_is_rejected():
    with pytest.raises(ValueError):
        riemann.star_state((1.0, -10.0, 0.1), (1.0, 10.0, 0.1))
