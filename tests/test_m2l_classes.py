"""The identity behind the FMM's M2L class products, checked on the CPU.

The reference's M2L (fast-multipole.cc:528-555) computes, for every pair,
    L_g(t) = 1/g! sum_a (-1)^|a| M_a(s) D_{g+a}(c_t - c_s)
with D_k = d^k (1/r). The GPU evaluates it per displacement class: cube
centres sit on a lattice, c_t - c_s = u v with u = min(h_t, h_s) and v an
integer vector, D is homogeneous (D_k(u v) = u^(-|k|-1) D_k(v)), and with
per-cell rescaled expansions
    Mh_a = (-1)^|a| M_a h_s^(-|a|),    L_g = h_t^(-|g|-1) Lh_g
a pair contributes Lh += A(v, d_t - d_s) Mh, where
    A[g][a] = 1/g! (h_t/u)^(|g|+1) (h_s/u)^|a| D_{g+a}(v)
depends on the class only. These tests restate both forms in numpy and
check that they agree for pairs at equal and different depths, with cube
centres built by repeated halving from a root half edge that is not a power
of two (as the octree builds them)."""
import math

import numpy as np
import pytest


def multi_indices(max_deg):
    """Multi-indices by degree, within a degree by a then b descending
    (fast-multipole.cc:41-178)."""
    out = []
    for deg in range(max_deg + 1):
        for a in range(deg, -1, -1):
            for b in range(deg - a, -1, -1):
                out.append((a, b, deg - a - b))
    return out


def derivatives(x, max_deg, index):
    """D_k(x) = d^k (1/|x|) for |k| <= max_deg by the recurrence
    r^2 D_k = -sum_j [(2 k_j - 1) x_j D_{k-e_j} + (k_j - 1)^2 D_{k-2e_j}]
    taken along the first nonzero axis, with the cross terms of the
    other axes (fast-multipole.cc:207-232)."""
    r2 = float(np.dot(x, x))
    mi = multi_indices(max_deg)
    D = np.zeros(len(mi))
    D[0] = 1.0 / math.sqrt(r2)
    for k, m in enumerate(mi[1:], start=1):
        i = 0 if m[0] > 0 else (1 if m[1] > 0 else 2)
        s = 0.0
        for j in range(3):
            dj = m[j]
            if dj == 0:
                continue
            t1 = list(m)
            t1[j] -= 1
            if j == i:
                s += (2 * dj - 1) * x[j] * D[index[tuple(t1)]]
                if dj >= 2:
                    t2 = list(t1)
                    t2[j] -= 1
                    s += (dj - 1) ** 2 * D[index[tuple(t2)]]
            else:
                s += 2.0 * dj * x[j] * D[index[tuple(t1)]]
                if dj >= 2:
                    t2 = list(t1)
                    t2[j] -= 1
                    s += dj * (dj - 1) * D[index[tuple(t2)]]
        D[k] = -s / r2
    return D


def cell(root_c, root_h, path):
    """Centre and half edge of the cube reached by halving along `path`
    (octant bits per level), as the octree builds them."""
    c = np.array(root_c, dtype=float)
    h = root_h
    for o in path:
        h *= 0.5
        c = c + h * np.array([1.0 if (o >> d) & 1 else -1.0 for d in range(3)])
    return c, h


@pytest.mark.parametrize("p", [2, 4])
def test_rescaled_class_form_equals_the_direct_contraction(p):
    rng = np.random.default_rng(7 + p)
    mi_d = multi_indices(2 * p)
    index = {m: k for k, m in enumerate(mi_d)}
    n_m = (p + 1) * (p + 2) * (p + 3) // 6
    mi = mi_d[:n_m]
    deg = np.array([sum(m) for m in mi])
    inv_fact = np.array([1.0 / (math.factorial(a) * math.factorial(b) * math.factorial(c)) for a, b, c in mi])
    sign = (-1.0) ** deg
    gpa = np.array([[index[(g[0] + a[0], g[1] + a[1], g[2] + a[2])] for a in mi] for g in mi])
    root_c, root_h = (0.013, -0.002, 0.004), 0.5 * (1 + 1e-9)
    checked = 0
    for trial in range(60):
        d_t = int(rng.integers(2, 6))
        d_s = int(np.clip(d_t + rng.integers(-2, 3), 1, 7))
        path_t = list(rng.integers(0, 8, d_t))
        path_s = list(rng.integers(0, 8, d_s))
        ct, ht = cell(root_c, root_h, path_t)
        cs, hs = cell(root_c, root_h, path_s)
        u = min(ht, hs)
        v = (ct - cs) / u
        rv = np.rint(v)
        assert np.max(np.abs(v - rv)) <= 1e-6  # centres on the lattice of the smaller cell
        if np.max(np.abs(rv)) < 3:  # well separated pairs only, as the acceptance test keeps them
            continue
        M = rng.normal(size=n_m) * hs ** deg  # a multipole of a cell of half edge hs
        # direct form
        D = derivatives(ct - cs, 2 * p, index)
        L_direct = inv_fact * ((sign * M)[None, :] * D[gpa]).sum(axis=1)
        # class form
        Dv = derivatives(rv, 2 * p, index)
        rt, rs = ht / u, hs / u  # powers of two
        assert rt == 2.0 ** round(math.log2(rt)) and rs == 2.0 ** round(math.log2(rs))
        A = (inv_fact * rt ** (deg + 1))[:, None] * (rs ** deg)[None, :] * Dv[gpa]
        Mh = sign * M * hs ** (-deg.astype(float))
        L_class = ht ** (-(deg + 1.0)) * (A @ Mh)
        scale = np.abs(inv_fact[:, None] * np.abs(M)[None, :] * np.abs(D[gpa])).sum(axis=1)
        assert np.all(np.abs(L_class - L_direct) <= 1e-12 * scale), (trial, d_t, d_s)
        checked += 1
    assert checked >= 20


def test_derivatives_are_homogeneous():
    p = 3
    mi_d = multi_indices(2 * p)
    index = {m: k for k, m in enumerate(mi_d)}
    deg = np.array([sum(m) for m in mi_d])
    v = np.array([3.0, -2.0, 5.0])
    D1 = derivatives(v, 2 * p, index)
    for u in (0.5, 0.125, 2.0 ** -20):
        Du = derivatives(u * v, 2 * p, index)
        np.testing.assert_allclose(Du, u ** (-(deg + 1.0)) * D1, rtol=1e-13, atol=0)


def test_derivatives_match_closed_forms():
    mi_d = multi_indices(4)
    index = {m: k for k, m in enumerate(mi_d)}
    x = np.array([0.3, -1.1, 0.7])
    r = np.linalg.norm(x)
    D = derivatives(x, 4, index)
    assert D[index[(1, 0, 0)]] == pytest.approx(-x[0] / r ** 3, rel=1e-14)
    assert D[index[(2, 0, 0)]] == pytest.approx((3 * x[0] ** 2 - r ** 2) / r ** 5, rel=1e-13)
    assert D[index[(1, 1, 0)]] == pytest.approx(3 * x[0] * x[1] / r ** 5, rel=1e-13)
    assert D[index[(1, 1, 1)]] == pytest.approx(-15 * x[0] * x[1] * x[2] / r ** 7, rel=1e-13)
    # Laplace: D_(2,0,0) + D_(0,2,0) + D_(0,0,2) = 0, and likewise one degree up
    assert abs(D[index[(2, 0, 0)]] + D[index[(0, 2, 0)]] + D[index[(0, 0, 2)]]) < 1e-13 / r ** 3
    assert abs(D[index[(3, 1, 0)]] + D[index[(1, 3, 0)]] + D[index[(1, 1, 2)]]) < 1e-12 / r ** 5


def test_derivatives_are_even_in_each_coordinate():
    # D_k(R w) = s^k D_k(w) for a reflection R = diag(s), s^k = prod_i s_i^k_i:
    # the identity that lets the tensor-core mode fold the 8 reflections of an
    # offset into one class
    p = 4
    mi_d = multi_indices(2 * p)
    index = {m: k for k, m in enumerate(mi_d)}
    w = np.array([3.0, 2.0, 5.0])
    Dw = derivatives(w, 2 * p, index)
    for R in range(8):
        s = np.array([-1.0 if (R >> i) & 1 else 1.0 for i in range(3)])
        sk = np.array([s[0] ** a * s[1] ** b * s[2] ** c for a, b, c in mi_d])
        np.testing.assert_allclose(derivatives(s * w, 2 * p, index), sk * Dw, rtol=1e-13, atol=0)


@pytest.mark.parametrize("p", [3, 5])
def test_reflected_class_matrix_is_the_signed_class_matrix_of_the_absolute_offset(p):
    # A(v) = S_g A(|v|) S_a: the product of a folded pair is the class product
    # of |v| with the source expansion taken with the signs s^a (the split
    # copy of reflection R) and row g multiplied by s^g afterwards
    mi_d = multi_indices(2 * p)
    index = {m: k for k, m in enumerate(mi_d)}
    n_m = (p + 1) * (p + 2) * (p + 3) // 6
    mi = mi_d[:n_m]
    deg = np.array([sum(m) for m in mi])
    inv_fact = np.array([1.0 / (math.factorial(a) * math.factorial(b) * math.factorial(c)) for a, b, c in mi])
    gpa = np.array([[index[(g[0] + a[0], g[1] + a[1], g[2] + a[2])] for a in mi] for g in mi])
    rng = np.random.default_rng(11 + p)
    for v in ([-3.0, 2.0, 4.0], [5.0, -1.0, -2.0], [-4.0, -4.0, 0.0], [0.0, 0.0, -3.0]):
        v = np.array(v)
        R = sum(1 << i for i in range(3) if v[i] < 0)
        s = np.array([-1.0 if (R >> i) & 1 else 1.0 for i in range(3)])
        sm = np.array([s[0] ** a * s[1] ** b * s[2] ** c for a, b, c in mi])
        rt, rs = 2.0, 1.0
        A_v = (inv_fact * rt ** (deg + 1))[:, None] * (rs ** deg)[None, :] * derivatives(v, 2 * p, index)[gpa]
        A_w = (inv_fact * rt ** (deg + 1))[:, None] * (rs ** deg)[None, :] * \
            derivatives(np.abs(v), 2 * p, index)[gpa]
        Mh = rng.normal(size=n_m)
        direct = A_v @ Mh
        folded = sm * (A_w @ (sm * Mh))
        np.testing.assert_allclose(folded, direct, rtol=1e-12, atol=1e-12 * np.abs(A_v).max())
