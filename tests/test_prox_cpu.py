"""The reference's unit tests of the constraints' proximal operators
(tests/cpd_test.c:129-300), run on the oracle's (orc_prox), plus the same
properties for the NTF regularizations, which the reference does not test.
No GPU, no reference build."""
import numpy as np

from oracles import PROX_KINDS as K


def _rand(shape, seed):
    return np.random.default_rng(seed).uniform(-3.0, 3.0, shape)


def test_nonneg(port):
    """cpd_test.c:129-154: every entry >= 0 after the prox."""
    v = _rand((10, 2), 1)
    v[0, 0] = -1.0
    assert (port.prox(K["nonneg"], v) >= 0.0).all()


def test_lasso_exact_values(port):
    """cpd_test.c:168-196: with multiplier 0.01 and rho 1, the entries 0.01,
    1.01 and -1.01 become exactly 0, 1 and -1."""
    mult = 0.01
    v = _rand((10, 2), 2)
    v.flat[0], v.flat[1], v.flat[2] = mult, 1.0 + mult, -1.0 - mult
    out = port.prox(K["lasso"], v, mult, 1.0)
    assert out.flat[0] == 0.0 and out.flat[1] == 1.0 and out.flat[2] == -1.0


def test_rowsimp_rows_on_simplex(port):
    """cpd_test.c:209-240: 100 x 11, every entry >= 0, every row sums to 1
    within 1e-6."""
    out = port.prox(K["rowsimp"], _rand((100, 11), 3), 0.0, 1.0)
    assert (out >= 0.0).all()
    assert np.abs(out.sum(axis=1) - 1.0).max() <= 1e-6


def test_colsimp_columns_on_simplex(port):
    """cpd_test.c:252-283: 100 x 11, every entry >= 0, every column sums to 1
    within 1e-6."""
    out = port.prox(K["colsimp"], _rand((100, 11), 4), 0.0, 1.0)
    assert (out >= 0.0).all()
    assert np.abs(out.sum(axis=0) - 1.0).max() <= 1e-6


def test_maxcolnorm(port):
    """maxcolnorm.c:32-62: columns of norm > 1 end at norm 1, the others are
    untouched; the non-negative form zeroes negatives first."""
    v = _rand((30, 6), 5)
    v[:, 2] *= 1e-2                                  # a column of norm < 1
    out = port.prox(K["maxcolnorm"], v)
    n = np.linalg.norm(out, axis=0)
    assert np.abs(n[[0, 1, 3, 4, 5]] - 1.0).max() <= 1e-12
    assert np.array_equal(out[:, 2], v[:, 2])
    nn = port.prox(K["maxcolnorm_nonneg"], v)
    assert (nn >= 0.0).all() and (np.linalg.norm(nn, axis=0) <= 1.0 + 1e-12).all()


def test_ntf_lasso_and_frob(port):
    """nonneg_lasso.c:29-45: v > L/rho -> v - L/rho, else 0; nonneg_frob.c:
    33-49: v rho / (L + rho), negatives zeroed."""
    L, rho = 0.5, 2.0
    v = np.array([[0.25, 0.3, -0.3, 1.25, 0.0]])
    thr, shrink = L / rho, rho / (L + rho)           # 0.25 and 0.8
    assert np.array_equal(port.prox(K["ntf_lasso"], v, L, rho),
                          [[0.0, 0.3 - thr, 0.0, 1.25 - thr, 0.0]])
    assert np.array_equal(port.prox(K["ntf_frob"], v, L, rho),
                          [[0.25 * shrink, 0.3 * shrink, 0.0, 1.25 * shrink, 0.0]])
