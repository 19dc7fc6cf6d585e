"""Oracle of the block GMRES (test infrastructure only: the tests import it
as the checker of rslab_gmres_block; the product never calls it).

A numpy restatement of the reference's right-preconditioned restarted block
GMRES, `gmres_block_mon` (src/numeric/iterative.rs:1908-2297), with its
helpers `givens` (:599-609), `well_conditioned_dim` (:624-639),
`finalize_block_column` (:1787-1830):
  * every cycle recomputes the live columns' true residuals and deflates
    those at tol (:2008-2055);
  * per step: block preconditioner apply, block operator apply, block
    classical Gram-Schmidt (:2075-2086) with a per-column second pass when a
    column's norm falls below 1/sqrt(2) of its norm before orthogonalisation
    (:2087-2118), Hessenberg column, Givens rotations, per-column
    convergence estimate |g_{j+1}| / ||b_c|| (:2119-2158);
  * columns that reach tol inside a cycle are finalised at once
    (x_c += M^-1 V_c y_c) and compacted out of the panel (:2159-2212);
  * the cycle ends with x_c += M^-1 (V_c y_c) for the columns still active
    (:2220-2262), and the final residuals of the columns never measured
    converged are recomputed (:2264-2284).
Vectors here are column-major n x s like the reference; projections are
plain numpy dot products (the reference folds 2048-row chunks), so
iteration counts may differ from the GPU's by one step, as the reference
itself notes for block vs single-vector GMRES.
"""
from __future__ import annotations

import numpy as np

EPS = np.finfo(np.float64).eps


def givens(f, g):
    if g == 0:
        return f * 0 + 1, g * 0
    if f == 0:
        return f * 0, g * 0 + 1
    r = np.sqrt(abs(f) ** 2 + abs(g) ** 2)
    return f / r, g / r


def well_conditioned_dim(h, jdim):
    if jdim == 0:
        return 0
    hmax = max(abs(h[i, i]) for i in range(jdim))
    th = EPS * hmax
    for i in range(jdim):
        if abs(h[i, i]) <= th:
            return i
    return jdim


def _backsub(h, g, jd):
    y = np.zeros(jd, dtype=h.dtype)
    for i in range(jd - 1, -1, -1):
        acc = g[i]
        for k in range(i + 1, jd):
            acc = acc - h[i, k] * y[k]
        y[i] = acc / h[i, i]
    return y


def gmres_block(apply_a, apply_m, b, tol, max_iter, restart, x0=None):
    """apply_a(X) / apply_m(R): n x k column blocks -> n x k.  b: n x s.
    Returns (x, iters, converged, final_res)."""
    b = np.asarray(b)
    n, s = b.shape
    dt = np.result_type(b.dtype, np.float64)
    m = max(restart, 1)
    x = np.zeros((n, s), dt) if x0 is None else np.array(x0, dt)
    bnorm = np.linalg.norm(b, axis=0)
    converged = bnorm == 0
    x[:, converged] = 0
    final_res = np.zeros(s)
    total = 0
    while total < max_iter:
        live = [c for c in range(s) if not converged[c]]
        if not live:
            break
        r_live = b[:, live] - apply_a(x[:, live])
        act, V0 = [], []
        h, g, cs, sn, jdim = [], [], [], [], []
        for a, c in enumerate(live):
            beta = np.linalg.norm(r_live[:, a])
            final_res[c] = beta / bnorm[c]
            if final_res[c] <= tol:
                converged[c] = True
                continue
            act.append(c)
            V0.append(r_live[:, a] / beta)
            h.append(np.zeros((m + 1, m), dt))
            gg = np.zeros(m + 1, dt)
            gg[0] = beta
            g.append(gg)
            cs.append(np.zeros(m, dt))
            sn.append(np.zeros(m, dt))
            jdim.append(0)
        sa = len(act)
        if sa == 0:
            break
        V = [np.stack(V0, axis=1)]  # V[j]: n x sa
        for j in range(m):
            if total >= max_iter:
                break
            w = apply_a(apply_m(V[j]))
            wn0 = np.linalg.norm(w, axis=0)
            p1 = np.array([[np.vdot(V[i][:, a], w[:, a]) for a in range(sa)] for i in range(j + 1)])
            for i in range(j + 1):
                w = w - V[i] * p1[i][None, :]
            reo = np.linalg.norm(w, axis=0) < (1 / np.sqrt(2)) * wn0
            p2 = np.zeros_like(p1)
            if reo.any():
                p2 = np.array([[np.vdot(V[i][:, a], w[:, a]) for a in range(sa)] for i in range(j + 1)])
                p2[:, ~reo] = 0
                for i in range(j + 1):
                    w = w - V[i] * p2[i][None, :]
            hn = np.linalg.norm(w, axis=0)
            V.append(np.where(hn > 0, w / np.where(hn > 0, hn, 1), 0))
            done = []
            for a in range(sa):
                H = h[a]
                H[: j + 1, j] = p1[:, a] + p2[:, a]
                H[j + 1, j] = hn[a]
                for i in range(j):
                    t = np.conj(cs[a][i]) * H[i, j] + np.conj(sn[a][i]) * H[i + 1, j]
                    H[i + 1, j] = -sn[a][i] * H[i, j] + cs[a][i] * H[i + 1, j]
                    H[i, j] = t
                c_, s_ = givens(H[j, j], H[j + 1, j])
                cs[a][j], sn[a][j] = c_, s_
                H[j, j] = np.conj(c_) * H[j, j] + np.conj(s_) * H[j + 1, j]
                H[j + 1, j] = 0
                g[a][j + 1] = -s_ * g[a][j]
                g[a][j] = np.conj(c_) * g[a][j]
                jdim[a] = j + 1
                if abs(g[a][j + 1]) / bnorm[act[a]] <= tol:
                    done.append(a)
            total += 1
            if done:
                for a in done:
                    jd = well_conditioned_dim(h[a], jdim[a])
                    if jd:
                        y = _backsub(h[a], g[a], jd)
                        vy = sum(V[i][:, a] * y[i] for i in range(jd))
                        x[:, act[a]] += apply_m(vy[:, None])[:, 0]
                keep = [a for a in range(sa) if a not in done]
                V = [Vi[:, keep] for Vi in V]
                h = [h[a] for a in keep]
                g = [g[a] for a in keep]
                cs = [cs[a] for a in keep]
                sn = [sn[a] for a in keep]
                jdim = [jdim[a] for a in keep]
                act = [act[a] for a in keep]
                sa = len(act)
                if sa == 0:
                    break
        if sa > 0:
            vy = np.zeros((n, sa), dt)
            for a in range(sa):
                jd = well_conditioned_dim(h[a], jdim[a])
                if jd:
                    y = _backsub(h[a], g[a], jd)
                    vy[:, a] = sum(V[i][:, a] * y[i] for i in range(jd))
            x[:, act] += apply_m(vy)
    pend = [c for c in range(s) if not converged[c] and bnorm[c] != 0]
    if pend:
        r = b[:, pend] - apply_a(x[:, pend])
        final_res[pend] = np.linalg.norm(r, axis=0) / bnorm[pend]
    final_res[bnorm == 0] = 0
    return x, total, bool(np.all(final_res <= tol)), final_res
