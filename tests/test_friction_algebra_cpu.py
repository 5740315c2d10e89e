"""CPU checks of the algebra the GPU friction solver relies on, against the
oracle's explicit 5N x 5N matrix (oracle/friction.py, src/SlipCalculator3D.jl:90-175):

  * the structured product: M v = [C u + (0; v4; v5); 2 mu v1 - v2; 2 mu v1 - v3]
    with u = [v1; v2 - mu v1; v3 - mu v1], and the transposed product, which
    csrc/lcp.cu evaluates instead of storing M;
  * the reduction of a Newton system J d = r (J = diag(Da) + diag(Db) M) to 3N
    unknowns by eliminating rows L4 / L5 element by element (solved for d4 / d5
    where |Da| >= |Db|, else for d2 / d3), which csrc/lcp.cu builds entry by
    entry from C: restated here in numpy and checked against the full solve;
  * the Fischer-Newton method on random P-matrix LCPs (unique solutions)."""
import numpy as np
import pytest
from hypothesis import given, settings
from hypothesis import strategies as st


def _case(seed, m):
    rng = np.random.default_rng(seed)
    C = rng.standard_normal((3 * m, 3 * m)) / np.sqrt(3 * m) + 2 * np.eye(3 * m)
    mu = rng.uniform(0, 0.8, m)
    Sf = rng.uniform(0, 1, m)
    b = rng.standard_normal(3 * m)
    return rng, C, mu, Sf, b


@pytest.mark.parametrize("seed,m", [(0, 7), (1, 30)])
def test_structured_products_match_explicit_matrix(seed, m):
    from oracle import friction as F
    rng, C, mu, Sf, b = _case(seed, m)
    M, q = F.friction_lcp(C, b, mu, Sf)
    v = rng.standard_normal(5 * m)
    v1, v2, v3, v4, v5 = (v[k * m:(k + 1) * m] for k in range(5))
    u = np.concatenate([v1, v2 - mu * v1, v3 - mu * v1])
    top = C @ u + np.concatenate([np.zeros(m), v4, v5])
    Mv = np.concatenate([top, 2 * mu * v1 - v2, 2 * mu * v1 - v3])
    assert np.allclose(Mv, M @ v, rtol=0, atol=1e-13 * np.abs(M @ v).max())
    s = C.T @ v[:3 * m]
    s1, s2, s3 = s[:m], s[m:2 * m], s[2 * m:]
    MTv = np.concatenate([s1 - mu * s2 - mu * s3 + 2 * mu * v4 + 2 * mu * v5, s2 - v4, s3 - v5, v2, v3])
    assert np.allclose(MTv, M.T @ v, rtol=0, atol=1e-13 * np.abs(M.T @ v).max())
    # the top of q is C (b - [0; Sf; Sf])
    assert np.allclose(q[:3 * m], C @ (b - np.concatenate([np.zeros(m), Sf, Sf])), rtol=0,
                       atol=1e-13 * np.abs(q).max())


def _reduced_direction(C, mu, m, Da, Db, r):
    """The 3N reduction of J d = r, restated from csrc/lcp.cu."""
    S = [slice(k * m, (k + 1) * m) for k in range(5)]
    a, bb, cc = {}, {}, {}
    for s, t in ((1, 3), (2, 4)):
        da, db, rt = Da[S[t]], Db[S[t]], r[S[t]]
        keep = np.abs(da) >= np.abs(db)          # row t solved for d_t
        one = np.ones(m)
        a[s] = np.where(keep, 0.0, -rt / np.where(keep, one, db))
        bb[s] = np.where(keep, 0.0, 2 * mu)
        cc[s] = np.where(keep, 1.0, da / np.where(keep, one, db))
        a[t] = np.where(keep, rt / np.where(keep, da, one), 0.0)
        bb[t] = np.where(keep, -2 * mu * db / np.where(keep, da, one), 0.0)
        cc[t] = np.where(keep, db / np.where(keep, da, one), 1.0)
    DbT = Db[:3 * m]
    CP = np.empty((3 * m, 3 * m))
    CP[:, S[0]] = C[:, S[0]] + C[:, S[1]] * (bb[1] - mu) + C[:, S[2]] * (bb[2] - mu)
    CP[:, S[1]] = C[:, S[1]] * cc[1]
    CP[:, S[2]] = C[:, S[2]] * cc[2]
    R = DbT[:, None] * CP
    rhs = r[:3 * m] - DbT * (C @ np.concatenate([np.zeros(m), a[1], a[2]]))
    idx = np.arange(m)
    R[idx, idx] += Da[S[0]]
    for s, t in ((1, 3), (2, 4)):
        R[s * m + idx, idx] += Da[S[s]] * bb[s] + Db[S[s]] * bb[t]
        R[s * m + idx, s * m + idx] += Da[S[s]] * cc[s] + Db[S[s]] * cc[t]
        rhs[S[s]] -= Da[S[s]] * a[s] + Db[S[s]] * a[t]
    v = np.linalg.solve(R, rhs)
    d = np.zeros(5 * m)
    d[S[0]] = v[S[0]]
    for s, t in ((1, 3), (2, 4)):
        d[S[s]] = a[s] + bb[s] * v[S[0]] + cc[s] * v[S[s]]
        d[S[t]] = a[t] + bb[t] * v[S[0]] + cc[t] * v[S[s]]
    return d


@pytest.mark.parametrize("seed,m", [(0, 12), (3, 40)])
def test_reduced_newton_system_matches_full_solve(seed, m):
    from oracle import friction as F
    rng, C, mu, Sf, b = _case(seed, m)
    M, q = F.friction_lcp(C, b, mu, Sf)
    n = 5 * m
    x = np.abs(rng.standard_normal(n)) * (rng.uniform(size=n) < 0.5)
    x[rng.uniform(size=n) < 0.1] = 0.0
    y = M @ x + q
    y[rng.choice(n, 3, replace=False)] = 0.0   # some rows with x = y = 0 (degenerate) as well
    phi = F.fb_phi(x, y)
    z = ((x == 0) & (y == 0)).astype(float)
    Da, Db = F.fb_jacobian_diag(x, y, z, M @ z)
    # every (Da, Db) lies on the circle (Da+1)^2 + (Db+1)^2 = 1: the pivot of the elimination is >= 1 - 1/sqrt(2)
    assert np.allclose((Da + 1) ** 2 + (Db + 1) ** 2, 1.0, atol=1e-14)
    assert np.maximum(np.abs(Da), np.abs(Db)).min() >= 1 - 1 / np.sqrt(2) - 1e-14
    J = Db[:, None] * M
    J[np.diag_indices(n)] += Da
    d_full = np.linalg.solve(J, -phi)
    d = _reduced_direction(C, mu, m, Da, Db, -phi)
    assert np.abs(d - d_full).max() <= 1e-12 * np.abs(d_full).max()


@settings(max_examples=25, deadline=None)
@given(seed=st.integers(0, 2 ** 31 - 1), n=st.integers(1, 25), act=st.floats(0.0, 1.0))
def test_fischer_newton_unique_solution_random(seed, n, act):
    from oracle import friction as F
    rng = np.random.default_rng(seed)
    R = rng.standard_normal((n, n))
    M = R @ R.T / n + np.eye(n)
    on = rng.uniform(size=n) < act
    xs = np.where(on, rng.uniform(0.5, 2.0, n), 0.0)
    ys = np.where(on, 0.0, rng.uniform(0.5, 2.0, n))
    q = ys - M @ xs
    x, it, rel = F.fischer_newton(M, q, tol=1e-12, max_iter=200)
    assert rel <= 1e-12
    assert np.abs(x - xs).max() <= 1e-9 * max(1.0, np.abs(xs).max())
