"""The su(3) algebra and exponential of the library against the identities of
the reference's ColorMatrixConstants::check (matrix-hmc.cpp:5-76), at its
bound qnorm < 1e-20 (qnorm = squared Frobenius norm):

- the generator T_a built from the unit basis vector e_a
  (set_anti_hermitian_matrix_from_basis) is traceless anti-Hermitian and
  projects back to e_a (set_basis_from_anti_hermitian_matrix);
- tr(T_a T_b) = -2 delta_ab;
- a momentum drawn by set_rand_gauge_momentum is traceless anti-Hermitian;
- with ad X from the basis projections of [X, T_b], the link update's
  exponential satisfies exp(c X) T_b exp(-c X) = sum_a exp(c ad X)_ab T_a
  (c = 0.2).

The reference's remaining checks concern the derivative of the exponential
map, which this library evaluates inside the flowed-HMC force; that force is
pinned against the reference library and finite differences in
tests/test_flowed_hmc.py.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GEO = (1, 1, 1, 32)  # 32 sites x 4 links: room for the 8 generators and 16 products


def qnorm(a):
    return float(np.sum(np.abs(a) ** 2))


def tr_less_anti_herm(m):
    a = 0.5 * (m - m.conj().T)
    return a - np.trace(a) / 3.0 * np.eye(3)


def expm(a, terms=40):
    r, t = np.eye(a.shape[0]), np.eye(a.shape[0])
    for k in range(1, terms):
        t = t @ a / k
        r = r + t
    return r


def generators(q, geo):
    """T_a from the unit basis vectors, through the library."""
    basis = np.zeros((32, 4 * 8))
    for a in range(8):
        basis[a, a] = 1.0  # site a, link 0, coefficient a
    b = q.FieldRealD(geo, 32)
    b.from_numpy(basis)
    fc = q.GaugeMomentum(geo)
    q.set_anti_hermitian_matrix_from_basis(fc, b)
    return np.asarray(fc)[:8, 0].copy(), fc, b


def project(q, geo, mats):
    """Basis coefficients of up to 32 anti-Hermitian matrices, through the library."""
    arr = np.zeros((32, 4, 3, 3), dtype=np.complex128)
    arr[:len(mats), 0] = mats
    fc = q.GaugeMomentum(geo)
    fc.from_numpy(arr)
    b = q.FieldRealD(geo, 32)
    q.set_basis_from_anti_hermitian_matrix(b, fc)
    return np.asarray(b.to_numpy()).reshape(32, 4, 8)[:len(mats), 0]


def test_generators(q):
    geo = q.Geometry(GEO)
    T, _, _ = generators(q, geo)
    for a in range(8):
        assert qnorm(tr_less_anti_herm(T[a]) - T[a]) < 1e-20
    proj = project(q, geo, T)
    assert qnorm(proj - np.eye(8)) < 1e-20
    for a in range(8):
        for b in range(8):
            tr = np.trace(T[a] @ T[b]) - (-2.0 if a == b else 0.0)
            assert abs(tr) ** 2 < 1e-20, (a, b, tr)


def test_exponential_conjugates_as_the_adjoint_exponential(q):
    geo = q.Geometry(GEO)
    T, _, _ = generators(q, geo)
    gm = q.GaugeMomentum(geo)
    gm.set_rand(q.RngState("ColorMatrixConstants::check"), 1.0)
    X = np.asarray(gm)[0, 0].copy()
    assert qnorm(X - tr_less_anti_herm(X)) < 1e-20
    # (ad X)_ab: coefficient of T_a in [X, T_b]
    adx = project(q, geo, np.array([X @ T[b] - T[b] @ X for b in range(8)])).T
    coef = 0.2
    exp_ad = expm(coef * adx)
    # exp(+c X) and exp(-c X) by the library's link update on unit links
    arr = np.zeros((32, 4, 3, 3), dtype=np.complex128)
    arr[:, :] = X
    p = q.GaugeMomentum(geo)
    p.from_numpy(arr)
    ex = {}
    for sign in (1, -1):
        u = q.GaugeField(geo)
        q.set_unit(u)
        q.gf_evolve(u, p, sign * coef)
        ex[sign] = np.asarray(u)[0, 0].copy()
    for b in range(8):
        mx_b = sum(exp_ad[a, b] * T[a] for a in range(8))
        assert qnorm(mx_b - ex[1] @ T[b] @ ex[-1]) < 1e-20, b
