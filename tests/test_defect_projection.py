"""The algebra of the projected defect correction (precision "mixed-dc"), restated in numpy.

A pressure matrix with setReference is A = L + c e_ref e_ref^T with L's rows summing to zero. The
device solves L y = r - (sum r) e_ref with the constant mode projected out, and corrects with
e = y + ((sum r) / c - y_ref) 1. These tests pin the identities that make that exact: the reference
row is the one row with a non-zero row sum, the right-hand side is compatible with L, and the
restored correction satisfies A e = r whatever constant the inner solution carries."""
import numpy as np

from voluma_b200 import mesh as vm


def dense(M, d, up):
    n = M["n_cells"]
    nI = M["n_internal_faces"]
    A = np.diag(d.astype(float))
    own, nei = M["owner"][:nI], M["neighbour"][:nI]
    A[own, nei] += up
    A[nei, own] += up
    return A


def test_reference_row_is_the_only_row_with_a_nonzero_sum():
    M = vm.box_mesh((6, 5, 4), hi=(1.0, 0.8, 0.9), periodic=(1, 0, 1))
    d, up = vm.poisson_matrix(M, ref_cell=7)
    A = dense(M, d, up)
    sums = A.sum(axis=1)
    big = np.abs(sums) > 1e-9 * np.abs(np.diag(A))
    assert np.flatnonzero(big).tolist() == [7]
    c = sums[7]
    L = A.copy()
    L[7, 7] -= c
    assert np.allclose(L.sum(axis=1), 0.0, atol=1e-12 * np.abs(np.diag(A)).max())


def test_restored_correction_solves_the_full_system():
    rng = np.random.default_rng(5)
    M = vm.box_mesh((5, 4, 6), hi=(1.0, 0.7, 1.1))
    d, up = vm.poisson_matrix(M, ref_cell=0)
    A = dense(M, d, up)
    c = A.sum(axis=1)[0]
    L = A.copy()
    L[0, 0] -= c
    r = rng.standard_normal(M["n_cells"])
    rhs = r.copy()
    rhs[0] -= r.sum()
    assert abs(rhs.sum()) < 1e-12 * np.abs(r).sum()  # compatible with L (1^T L = 0)
    # any solution of L y = rhs: least squares picks one, then an arbitrary constant is added
    y = np.linalg.lstsq(L, rhs, rcond=None)[0] + 3.7
    assert np.allclose(L @ y, rhs, atol=1e-10)
    e = y + (r.sum() / c - y[0])
    assert np.allclose(A @ e, r, atol=1e-10)
    assert np.allclose(e, np.linalg.solve(A, r), atol=1e-9)


def test_projected_preconditioned_residual_keeps_the_dot():
    """wArA = (z - mean z) . r equals z . r - mean(z) sum(r), the form the inner dot kernel uses."""
    rng = np.random.default_rng(6)
    z = rng.standard_normal(100)
    r = rng.standard_normal(100)
    mu = z.mean()
    assert np.isclose((z - mu) @ r, z @ r - mu * r.sum())
