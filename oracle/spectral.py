"""GLL / GLJ tables for nPol = 4, from their definitions (test infrastructure).

The reference hard-codes these tables rounded to 12 decimals in
SOLVER/src/preloop/se_model/quad/spectrals.hpp:73-102 (the ``_NPOL == 4`` block).
Here they are derived from the mathematics and rounded the same way; the pin
test (tests/test_oracle_pins.py) compares them with the reference's values,
extracted as text into tests/golden/spectral_npol4.json.

* GLL nodes: -1, +1 and the roots of P_4'(x) (Legendre).
* GLJ nodes (axial direction xi, weight 1 + xi): -1, +1 and the roots of the
  Jacobi polynomial P_3^(1,2)(x).
* weights: exact quadrature of degree <= 2N-1 under the respective weight.
* G matrices: G(j, i) = l_j'(x_i) for the Lagrange basis on the nodes
  (``gGMatrixGLL`` / ``gGMatrixGLJ``, row-major).
"""
import numpy as np
from numpy.polynomial import legendre
from scipy.special import roots_jacobi

NPOL = 4
NPED = NPOL + 1


def _round12(x):
    return np.round(np.asarray(x, dtype=np.float64), 12) + 0.0


def nodes_gll():
    c = np.zeros(NPED)
    c[-1] = 1.0
    inner = np.sort(legendre.legroots(legendre.legder(c)).real)
    return np.concatenate([[-1.0], inner, [1.0]])


def nodes_glj():
    inner, _ = roots_jacobi(NPOL - 1, 1.0, 2.0)
    return np.concatenate([[-1.0], np.sort(inner), [1.0]])


def _weights(x, weight_moments):
    # solve sum_i w_i x_i^k = int w(x) x^k dx, k = 0..N
    V = np.vander(x, NPED, increasing=True).T
    return np.linalg.solve(V, weight_moments)


def weights_gll():
    k = np.arange(NPED)
    mom = np.where(k % 2 == 0, 2.0 / (k + 1), 0.0)
    return _weights(nodes_gll(), mom)


def weights_glj():
    # int_{-1}^{1} (1 + x) x^k dx
    k = np.arange(NPED)
    mom = np.where(k % 2 == 0, 2.0 / (k + 1), 0.0) + np.where(k % 2 == 1, 2.0 / (k + 2), 0.0)
    return _weights(nodes_glj(), mom)


def lagrange_deriv_matrix(x):
    """G[j, i] = l_j'(x_i)."""
    n = len(x)
    G = np.zeros((n, n))
    for j in range(n):
        for i in range(n):
            s = 0.0
            for m in range(n):
                if m == j:
                    continue
                prod = 1.0 / (x[j] - x[m])
                for k in range(n):
                    if k in (j, m):
                        continue
                    prod *= (x[i] - x[k]) / (x[j] - x[k])
                s += prod
            G[j, i] = s
    return G


def lagrange_weights(x, xi):
    """l_j(xi) for all j (SE_Model::computeInplaneFactor uses these)."""
    n = len(x)
    w = np.ones(n)
    for j in range(n):
        for k in range(n):
            if k != j:
                w[j] *= (xi - x[k]) / (x[j] - x[k])
    return w


def tables():
    """The tables as the reference stores them (rounded to 12 decimals)."""
    return {
        "pGLL": _round12(nodes_gll()),
        "pGLJ": _round12(nodes_glj()),
        "wGLL": _round12(weights_gll()),
        "wGLJ": _round12(weights_glj()),
        "gGLL": _round12(lagrange_deriv_matrix(nodes_gll())).ravel(),
        "gGLJ": _round12(lagrange_deriv_matrix(nodes_glj())).ravel(),
    }
