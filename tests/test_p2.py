"""The p = 2 modal basis on the CPU: the reference-element tables the kernels use
(dgr_p2_reference) against the basis' defining properties."""
from __future__ import annotations

import numpy as np


def test_basis_is_orthogonal_with_the_closed_form_norms(dgrain):
    R = dgrain.p2.reference()
    G = (R["phi"].T * (2 * R["wq"])) @ R["phi"]  # the degree-5 rule is exact for these degree-4 products
    np.testing.assert_allclose(G, np.diag(np.diag(G)), atol=1e-14)
    # int over the reference triangle of phi_ij^2 = 2 / ((2i+1)(i+j+1)) in the hierarchical
    # order (0,0), (0,1), (1,0), (0,2), (1,1), (2,0)
    ij = [(0, 0), (0, 1), (1, 0), (0, 2), (1, 1), (2, 0)]
    want = [2.0 / ((2 * i + 1) * (i + j + 1)) for i, j in ij]
    np.testing.assert_allclose(R["mass"], want, rtol=1e-14)
    np.testing.assert_allclose(np.diag(G), want, rtol=1e-14)


def test_rule_and_gauss_points(dgrain):
    R = dgrain.p2.reference()
    assert abs(R["wq"].sum() - 1.0) < 1e-15 and abs(R["wg"].sum() - 2.0) < 1e-15
    # the area rule integrates x^a y^b exactly up to degree 5 (reference triangle)
    r, s = R["rs"][:, 0], R["rs"][:, 1]
    for a, b, exact in ((0, 0, 2.0), (1, 0, -2.0 / 3), (2, 0, 2.0 / 3), (2, 2, 2.0 / 9)):
        assert abs(2 * (R["wq"] * r ** a * s ** b).sum() - exact) < 1e-14, (a, b)
    # basis at the edge Gauss points = basis at the mapped reference coordinates
    t = R["te"]
    for k, (rr, ss) in enumerate(((t, -np.ones(3)), (-t, t), (-np.ones(3), -t))):
        A, B = rr + (1 + ss) / 2, (1 - ss) / 2
        phi = np.stack([np.ones(3), (3 * ss + 1) / 2, A, (5 * ss ** 2 + 2 * ss - 1) / 2, A * (5 * ss + 3) / 2,
                        (3 * A ** 2 - B ** 2) / 2], axis=1)
        np.testing.assert_allclose(R["phie"][k], phi, atol=1e-15)


def test_projection_is_exact_for_quadratics(dgrain):
    m = dgrain.rectangle(6, 3, jitter=0.2, seed=1)
    f = lambda x, y: 1 + 2 * x / 1e4 - 3 * y / 1e4 + (x / 1e4) ** 2 - x * y / 1e8 + 0.5 * (y / 1e4) ** 2  # noqa
    c = dgrain.p2.project(m, f)
    assert dgrain.p2.l2_error(m, c, f) <= 1e-11 * np.sqrt(1e4 * 5e3)
    assert abs(dgrain.p2.volume(m, dgrain.p2.project(m, lambda x, y: np.ones_like(x))) - 5e7) < 1e-6


def test_gauge_weights_are_the_basis_at_the_point(dgrain):
    """p2.gauge_weights evaluates the basis at a physical point: at an element's area
    quadrature points it reproduces the kernels' table, and the modal elevation there"""
    m = dgrain.rectangle(6, 3, jitter=0.2, seed=4)
    R = dgrain.p2.reference()
    np.testing.assert_allclose(dgrain.p2.basis(R["rs"][:, 0], R["rs"][:, 1]), R["phi"], atol=1e-15)
    X, Y, _ = dgrain.p2.quadrature_points(m, R)
    e = 7
    el, w = dgrain.p2.gauge_weights(m, list(zip(X[e], Y[e])))
    assert (el == e).all()
    np.testing.assert_allclose(w, R["phi"], atol=1e-12)
    c = dgrain.p2.project(m, lambda x, y: 1 + x / 1e4 - (y / 1e4) ** 2)
    np.testing.assert_allclose((w * c.reshape(-1, 6)[el]).sum(axis=1), dgrain.p2.evaluate(m, c, R)[e], atol=1e-12)
