"""The compact Roe form of the face Jacobians, as algebra on the CPU.

An inviscid face Jacobian `area * K` (physics.cuh:roe_k_matrix, after
fluxInviscid.loci:1019-1090) is spanned by nine direction coefficients
with the area folded in (a1 = A l1 rT, c7, c8, c4, c1, lr = A l1 rho,
l9 = A l1 c9, c10, c11), plus the face's Roe velocity U and normal n.
The assembly expands them entry by entry (compact_expand). The sweeps
apply them in factored form (compact_apply):

    y0  = a1 x0 + c7 dun + c8 x4
    y_r = U_r y0 + n_r (c4 dun - c1 x4) + lr x_r
    y4  = l9 x0 + c10 dun + lr U.x_m + c11 x4

This test restates both in numpy. It checks that the factored product
equals the product with the 25-entry matrix, which is the matrix
roe_k_matrix spells out. CPU only.
"""
import numpy as np


def expand(c, U, n):
    """the 25 entries of roe_k_matrix, from the compact coefficients"""
    a1, c7, c8, c4, c1, lr, l9, c10, c11 = c
    M = np.zeros((5, 5))
    M[0, 0] = a1
    M[0, 1:4] = n * c7
    M[0, 4] = c8
    for r in range(3):
        M[1 + r, 0] = a1 * U[r]
        M[1 + r, 1:4] = n * (c7 * U[r] + n[r] * c4)
        M[1 + r, 1 + r] += lr
        M[1 + r, 4] = c8 * U[r] - n[r] * c1
    M[4, 0] = l9
    M[4, 1:4] = n * c10 + lr * U
    M[4, 4] = c11
    return M


def apply(c, U, n, x):
    a1, c7, c8, c4, c1, lr, l9, c10, c11 = c
    dun = n @ x[1:4]
    y0 = a1 * x[0] + c7 * dun + c8 * x[4]
    w = c4 * dun - c1 * x[4]
    y = np.empty(5)
    y[0] = y0
    y[1:4] = U * y0 + n * w + lr * x[1:4]
    y[4] = l9 * x[0] + c10 * dun + lr * (U @ x[1:4]) + c11 * x[4]
    return y


def test_factored_product_equals_the_matrix_product():
    rng = np.random.default_rng(7)
    for _ in range(200):
        c = rng.standard_normal(9) * 10.0 ** rng.uniform(-3, 3, 9)
        U = rng.standard_normal(3) * 300.0
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        x = rng.standard_normal(5)
        M = expand(c, U, n)
        y = apply(c, U, n, x)
        ref = M @ x
        scale = np.abs(M).max() * np.abs(x).max()
        assert np.abs(y - ref).max() <= 1e-12 * scale


def test_negated_coefficients_negate_the_matrix():
    """a lower slot stores L = -fjp by negating the nine coefficients"""
    rng = np.random.default_rng(8)
    c, U = rng.standard_normal(9), rng.standard_normal(3)
    n = rng.standard_normal(3)
    n /= np.linalg.norm(n)
    np.testing.assert_array_equal(expand(-c, U, n), -expand(c, U, n))


def test_wall_block_is_the_pressure_column():
    """a viscous-wall face keeps only d(p n A)/dpg: c1 = -A, the rest zero"""
    A, n, U = 0.3, np.array([0.0, 0.6, 0.8]), np.array([1.0, 2.0, 3.0])
    c = np.zeros(9)
    c[4] = -A
    M = expand(c, U, n)
    ref = np.zeros((5, 5))
    ref[1:4, 4] = n * A
    np.testing.assert_array_equal(M, ref)
