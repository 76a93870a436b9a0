"""Host pieces of the adjoint: the Kepler Jacobians (no GPU)."""

import numpy as np

from sailfish_b200.adjoint import mass_jacobian, mass_jacobians


def test_vectorised_kepler_jacobian_matches_the_scalar_one():
    times = np.array([0.0, 0.37, 1.9, 6.4, 12.7, 40.03])
    for q, e in ((0.5, 0.1), (1.0, 0.0), (0.2, 0.6)):
        many = mass_jacobians(times, q, e)
        assert many.shape == (len(times), 10, 2)
        for t, jac in zip(times, many):
            np.testing.assert_allclose(jac, mass_jacobian(t, q, e), rtol=1e-13, atol=1e-15)


def test_kepler_jacobian_matches_central_differences():
    from sailfish_b200.adjoint import _kepler_complex

    t, q, e, h = 2.3, 0.5, 0.1, 1e-6
    jac = mass_jacobians(np.array([t]), q, e)[0]
    for col, (dq, de) in enumerate(((h, 0.0), (0.0, h))):
        plus = np.array([v.real for v in _kepler_complex(t, 1.0, 1.0, complex(q + dq), complex(e + de))])
        minus = np.array([v.real for v in _kepler_complex(t, 1.0, 1.0, complex(q - dq), complex(e - de))])
        np.testing.assert_allclose(jac[:, col], (plus - minus) / (2 * h), rtol=1e-6, atol=1e-8)
