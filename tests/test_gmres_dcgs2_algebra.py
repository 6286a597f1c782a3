"""The device GMRES's Arnoldi step (delayed classical Gram-Schmidt with
re-orthogonalisation, solvers.cu `gmres`) restated in numpy, step for step as
the host logic runs it, against textbook GMRES with modified Gram-Schmidt:
the same iteration counts, the same residual estimates and an orthonormal
basis.  CPU only."""
import numpy as np


def _rotate(Hr, cs, sn, g, jc):
    """Givens rotations of column jc (previous ones, then its own); returns
    the new residual estimate |g[jc + 1]|."""
    for i in range(jc):
        a, c = Hr[i, jc], Hr[i + 1, jc]
        Hr[i, jc], Hr[i + 1, jc] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
    a, c = Hr[jc, jc], Hr[jc + 1, jc]
    rr = np.hypot(a, c)
    cs[jc], sn[jc] = a / rr, c / rr
    Hr[jc, jc], Hr[jc + 1, jc] = rr, 0.0
    g[jc + 1], g[jc] = -sn[jc] * g[jc], cs[jc] * g[jc]
    return abs(g[jc + 1])


def _lsq_update(x, V, Hr, g, k):
    y = np.zeros(k)
    for i in range(k - 1, -1, -1):
        y[i] = (g[i] - Hr[i, i + 1:k] @ y[i + 1:k]) / Hr[i, i]
    return x + y @ V[:k]


def gmres_dcgs2(A, b, m, tol, max_it):
    """Returns (x, iterations, estimates per iteration, worst orthogonality loss)."""
    n = len(b)
    x, it, tolabs, est, orth = np.zeros(n), 0, None, [], 0.0
    while True:
        r = b - A @ x
        beta = np.linalg.norm(r)
        tolabs = tol * beta if tolabs is None else tolabs
        if beta <= tolabs or it >= max_it:
            return x, it, est, orth
        V = np.zeros((m + 1, n))
        V[0] = r / beta
        H, Hr = np.zeros((m + 1, m)), np.zeros((m + 1, m))
        cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
        g[0] = beta
        it0, k, done, j = it, 0, False, 0
        while True:
            last = j == m or it0 + j >= max_it
            if not last:
                V[j + 1] = A @ V[j]                      # w = B u_j
            hs = V[:j + 1] @ V[j]                        # Q^T u_j and u_j.u_j
            hz = V[:j + 1] @ V[j + 1] if not last else None
            ss, t = hs[:j] @ hs[:j], hs[j]
            sz = hs[:j] @ hz[:j] if not last else 0.0
            alpha = np.sqrt(t - ss) if t - ss > 1e-28 * t else 0.0
            if j > 0:                                    # column j-1 is final
                H[:j, j - 1] += hs[:j]
                H[j, j - 1] = alpha
                Hr[:j + 1, j - 1] = H[:j + 1, j - 1]
                it += 1
                est.append(_rotate(Hr, cs, sn, g, j - 1))
                if est[-1] <= tolabs:
                    k, done = j, True
                    break
            if last or alpha == 0.0:
                k = j
                break
            ia = 1.0 / alpha
            c = np.append(hz[:j] * ia, (hz[j] - sz) * ia * ia)
            for i in range(j + 1):
                H[i, j] = c[i] - sum(H[i, l] * hs[l] for l in range(max(0, i - 1), j)) * ia
            q = (V[j] - hs[:j] @ V[:j]) * ia             # the sweep
            V[j + 1] = V[j + 1] * ia - c[:j] @ V[:j] - c[j] * q
            V[j] = q
            j += 1
        if k > 0:
            x = _lsq_update(x, V, Hr, g, k)
            orth = max(orth, np.abs(V[:k] @ V[:k].T - np.eye(k)).max())
        if done or it >= max_it:
            return x, it, est, orth


def gmres_mgs(A, b, m, tol, max_it):
    n = len(b)
    x, it, tolabs, est = np.zeros(n), 0, None, []
    while True:
        r = b - A @ x
        beta = np.linalg.norm(r)
        tolabs = tol * beta if tolabs is None else tolabs
        if beta <= tolabs or it >= max_it:
            return x, it, est
        V, Hr = np.zeros((m + 1, n)), np.zeros((m + 1, m))
        cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
        V[0], g[0] = r / beta, beta
        for j in range(m):
            w = A @ V[j]
            for i in range(j + 1):
                Hr[i, j] = w @ V[i]
                w -= Hr[i, j] * V[i]
            Hr[j + 1, j] = np.linalg.norm(w)
            V[j + 1] = w / Hr[j + 1, j]
            it += 1
            est.append(_rotate(Hr, cs, sn, g, j))
            if est[-1] <= tolabs or it >= max_it:
                break
        x = _lsq_update(x, V, Hr, g, j + 1)
        if est[-1] <= tolabs:
            return x, it, est


def _systems():
    rng = np.random.default_rng(1)
    n = 240
    yield "near identity", np.eye(n) + 0.3 * rng.standard_normal((n, n)) / np.sqrt(n), rng.standard_normal(n)
    # 1D convection-diffusion stencil: slow, restarted convergence
    A = np.diag(np.full(n, 2.0)) + np.diag(np.full(n - 1, -1.3), -1) + np.diag(np.full(n - 1, -0.7), 1)
    yield "convection-diffusion", A, rng.standard_normal(n)


def test_dcgs2_matches_modified_gram_schmidt():
    for name, A, b in _systems():
        for m in (30, 7):
            x, it, est, orth = gmres_dcgs2(A, b, m, 1e-10, 150)
            xr, itr, estr = gmres_mgs(A, b, m, 1e-10, 150)
            assert it == itr, (name, m, it, itr)
            e, er = np.array(est), np.array(estr)
            assert np.all(np.abs(e - er) <= 1e-8 * er + 1e-12 * er[0]), (name, m)
            assert orth < 1e-13, (name, m, orth)
            assert np.linalg.norm(x - xr) <= 1e-8 * np.linalg.norm(xr), (name, m)


def test_dcgs2_converges_to_tolerance():
    name, A, b = next(_systems())
    x, it, est, _ = gmres_dcgs2(A, b, 30, 1e-10, 500)
    assert est[-1] <= 1e-10 * np.linalg.norm(b)
    assert np.linalg.norm(b - A @ x) <= 2e-10 * np.linalg.norm(b)
