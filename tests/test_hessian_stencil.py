"""Host Hessian from gradient differences against the reference's
sum_gradient / sum_hessian known answer (``tf_pwa/tests/test_model_new.py:7-20``):
f(a, b) = sum over batches x in [1, 2] of a + b^2 + x at a = 1, b = 2 gives
nll 13, gradient [2, 8], Hessian [[0, 0], [0, 4]]."""
import numpy as np


def _batched(x):
    a, b = x
    nll = sum(a + b ** 2 + xb for xb in (1.0, 2.0))
    return nll, np.array([2.0, 2 * 2 * b])


def test_sum_hessian_known_answer():
    from tf_pwa_b200.api import hessian_from_gradient

    for step in (1e-4, 1e-2):
        nll, g, h = hessian_from_gradient(_batched, [1.0, 2.0], step)
        assert nll == 13.0
        np.testing.assert_allclose(g, [2.0, 8.0])
        np.testing.assert_allclose(h, [[0.0, 0.0], [0.0, 4.0]], atol=1e-9)


def test_stencil_exact_for_quartic():
    """A quartic f has a cubic gradient: the 4-point stencil reproduces its
    Hessian up to rounding."""
    from tf_pwa_b200.api import hessian_from_gradient

    def f(x):
        u, v = x
        val = u ** 4 + 3 * u * u * v - v ** 3 + 2 * u * v
        g = np.array([4 * u ** 3 + 6 * u * v + 2 * v, 3 * u * u - 3 * v * v + 2 * u])
        return val, g

    x = np.array([0.7, -1.3])
    u, v = x
    exact = np.array([[12 * u * u + 6 * v, 6 * u + 2], [6 * u + 2, -6 * v]])
    _, _, h = hessian_from_gradient(f, x, 1e-2)
    np.testing.assert_allclose(h, exact, rtol=1e-10, atol=1e-10)
