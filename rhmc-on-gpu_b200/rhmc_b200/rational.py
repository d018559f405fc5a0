"""Rational approximations r(x) = a0 + sum_i a_i / (x + b_i) of x^p on [eps, 1].

The reference builds them at start-up with AlgRemez over MPFR (lib/Tools/RationalApprox/
rationalapprox_calc.cc:8-177, alg_remez.cc) and stores them normalised on [lambda_min, 1] in a
RationalApprox (rationalapprox.h:13-47); the first/md/last coefficients are then rescaled by the
largest eigenvalue (rationalapprox.cc:134-266).  MPFR is not available here, so this module
produces the same object a different way: poles b_i > 0 are placed log-uniformly (the sinc
quadrature of x^-q = sin(pi q)/pi int_0^inf t^-q/(t+x) dt), the numerators follow from a linear
least-squares fit of the relative error on a log grid, and the log-poles are then adjusted with
scipy's least_squares to minimise the relative error, which approaches the minimax (Remez)
solution.  For 0 < p < 1 the form x * x^(p-1) gives a0 = sum w_i and a_i = -w_i b_i.

The result is returned with its measured maximum relative error on [eps, 1]; the oracle and the
GPU path read the same numbers, so approximation quality does not affect parity.
"""
import numpy as np


def _design(x, b, with_a0):
    cols = [1.0 / (x[:, None] + b[None, :])]
    if with_a0:
        cols.insert(0, np.ones((x.size, 1)))
    return np.hstack(cols)


def _fit(x, f, b, with_a0):
    A = _design(x, b, with_a0) / f[:, None]
    coef, *_ = np.linalg.lstsq(A, np.ones_like(f), rcond=None)
    return coef


def _eval(x, b, coef, with_a0):
    return _design(x, b, with_a0) @ coef


def inverse_power(q, n, eps, optimise=True, grid=3000):
    """x^-q (0 < q < 1) on [eps, 1] with n poles: a0 = 0."""
    x = np.geomspace(eps, 1.0, grid)
    f = x ** (-q)
    # sinc-quadrature pole positions: log-uniform a little beyond the interval
    lo, hi = np.log(eps) - 2.0, np.log(1.0) + 3.0
    s = np.linspace(lo, hi, n)
    b = np.exp(s)

    def resid(logb):
        bb = np.exp(logb)
        c = _fit(x, f, bb, False)
        return _eval(x, bb, c, False) / f - 1.0

    if optimise and n > 1:
        from scipy.optimize import least_squares
        # keep the poles within a few decades of the interval (a pole running off to infinity
        # only mimics a constant term and makes a useless solver shift)
        blo, bhi = np.log(eps) - 6.0, np.log(1.0) + 6.0
        sol = least_squares(resid, np.clip(s, blo + 1e-9, bhi - 1e-9), bounds=(blo, bhi), method="trf", max_nfev=3000)
        s = np.sort(sol.x)
        b = np.exp(s)
    a = _fit(x, f, b, False)
    err = np.max(np.abs(_eval(x, b, a, False) / f - 1.0))
    return 0.0, a, b, err


def rational_power(p, n, eps, optimise=True, method="minimax"):
    """Coefficients of x^p on [eps, 1], p in (-1, 0) or (0, 1), degree n.
    Returns dict(a0, a, b, min_eps, power, max_rel_err).  method "minimax" (default):
    minimax_power (type (n, n), near-minimax relative error, the kind of approximation the
    reference's AlgRemez produces, rationalapprox_calc.cc:8-177); "lsq": the pole-optimised least
    squares fit above (a0 = 0 for negative powers), usually orders of magnitude less accurate at
    the same degree."""
    if method == "minimax":
        try:
            return minimax_power(p, n, eps)
        except ValueError as e:
            if not (0.0 < abs(p) < 1.0):
                raise
            # AAA finds spurious pole pairs when n is far more than the power needs (x^(1/32)
            # with 20 poles); the least-squares fit keeps n real negative poles there
            out = rational_power(p, n, eps, optimise, method="lsq")
            out["method"] = "lsq (minimax: %s)" % e
            return out
    if method != "lsq":
        raise ValueError("method must be 'lsq' or 'minimax'")
    if 0.0 < -p < 1.0:
        a0, a, b, err = inverse_power(-p, n, eps, optimise)
    elif 0.0 < p < 1.0:
        # x^p = x * x^(p-1):  x sum w/(x+b) = sum w - sum w b/(x+b)
        _, w, b, _ = inverse_power(1.0 - p, n, eps, optimise)
        a0 = float(np.sum(w))
        a = -w * b
        x = np.geomspace(eps, 1.0, 3000)
        r = a0 + (a[None, :] / (x[:, None] + b[None, :])).sum(1)
        err = float(np.max(np.abs(r / x ** p - 1.0)))
    else:
        raise ValueError("power must be in (-1, 0) or (0, 1)")
    return {"a0": float(a0), "a": [float(v) for v in a], "b": [float(v) for v in b], "min_eps": float(eps),
            "power": float(p), "max_rel_err": float(err)}


def rescale(approx, lam_max, exponent):
    """The rescaling of RationalApprox::*_inv_approx_coeff (rationalapprox.cc:162-170, 206-214,
    250-258): with e = lam_max^exponent, a0 -> a0 e, a_i -> a_i lam_max e, b_i -> b_i lam_max.
    lam_max is the already enlarged bound (the reference multiplies findminmax's max by 1.05)."""
    e = lam_max ** exponent
    return {"a0": approx["a0"] * e, "a": [v * lam_max * e for v in approx["a"]], "b": [v * lam_max for v in approx["b"]]}


def _aaa_lawson(x, f, m, lawson):
    """Barycentric rational r(x) = sum_j w_j f_j/(x - z_j) / sum_j w_j/(x - z_j) of type
    (m-1, m-1) minimising the relative error |r/f - 1| on the points x: AAA (Nakatsukasa, Sete and
    Trefethen, SIAM J. Sci. Comput. 40 (2018) A1494) picks the support points z_j greedily, then
    Lawson's iteratively reweighted least squares (Nakatsukasa and Trefethen, SIAM J. Sci. Comput.
    42 (2020) A3157) moves the weights towards the minimax solution.  Returns (z, f_z, w, err)."""
    rest = np.ones(len(x), bool)
    r = np.full_like(f, np.mean(f))
    z, fz = [], []
    for _ in range(m):
        e = np.where(rest, np.abs(r / f - 1.0), -1.0)
        j = int(np.argmax(e))
        z.append(x[j])
        fz.append(f[j])
        rest[j] = False
        zz, ff = np.array(z), np.array(fz)
        C = 1.0 / (x[rest][:, None] - zz[None, :])
        A = (f[rest][:, None] - ff[None, :]) * C / f[rest][:, None]  # linearised relative error
        w = np.linalg.svd(A, full_matrices=False)[2][-1]
        r = f.copy()
        r[rest] = (C @ (w * ff)) / (C @ w)
    zz, ff = np.array(z), np.array(fz)
    C = 1.0 / (x[rest][:, None] - zz[None, :])
    A = (f[rest][:, None] - ff[None, :]) * C / f[rest][:, None]
    wt = np.full(A.shape[0], 1.0 / A.shape[0])
    best = (np.inf, None)
    for _ in range(lawson):
        w = np.linalg.svd(np.sqrt(wt)[:, None] * A, full_matrices=False)[2][-1]
        e = np.abs((C @ (w * ff)) / (C @ w) / f[rest] - 1.0)
        if e.max() < best[0]:
            best = (e.max(), w.copy())
        wt = wt * e
        wt /= wt.sum()
    return zz, ff, best[1], best[0]


def _bary_poles(z, w):
    """Poles of a barycentric rational: the finite eigenvalues of the pencil
    ([0 w^T; 1 diag(z)], diag(0, 1, ..., 1))."""
    from scipy.linalg import eig
    m = len(z)
    E = np.zeros((m + 1, m + 1))
    E[0, 1:] = w
    E[1:, 0] = 1.0
    E[1:, 1:] = np.diag(z)
    B = np.eye(m + 1)
    B[0, 0] = 0.0
    ev = eig(E, B, right=False)
    return ev[np.isfinite(ev)]


def minimax_power(p, n, eps, grid=4000, lawson=150):
    """x^p on [eps, 1], p in (-1, 0) or (0, 1), as a0 + sum_i a_i/(x + b_i) with n poles: a
    near-minimax approximation of type (n, n) in the relative error (the kind the reference's
    AlgRemez produces, rationalapprox_calc.cc:8-177), from AAA-Lawson.  The poles are the
    barycentric form's (all real and negative for these powers; anything else raises
    ValueError); the numerators are then taken from the barycentric form or from a least-squares
    fit of the relative error, whichever has the smaller maximum error on a 4x finer grid.
    Returns the dictionary of rational_power."""
    if not (0.0 < abs(p) < 1.0):
        raise ValueError("power must be in (-1, 0) or (0, 1)")
    x = np.geomspace(eps, 1.0, grid)
    f = x ** p
    z, fz, w, _ = _aaa_lawson(x, f, n + 1, lawson)
    pol = _bary_poles(z, w)
    if len(pol) != n or np.any(np.abs(pol.imag) > 1e-9 * np.abs(pol)) or np.any(pol.real >= 0.0):
        raise ValueError("the approximation of x^%g with %d poles has poles off the negative real axis" % (p, n))
    b = np.sort(-pol.real)
    xf = np.geomspace(eps, 1.0, 4 * grid)
    ffine = xf ** p
    # numerators from the barycentric form: a0 = r(inf), a_i = N(-b_i) / D'(-b_i)
    N = lambda t: np.sum(w * fz / (t - z))
    dD = lambda t: -np.sum(w / (t - z) ** 2)
    cand = [np.concatenate([[np.sum(w * fz) / np.sum(w)], [N(-bi) / dD(-bi) for bi in b]]),
            _fit(xf, ffine, b, True)]
    errs = [np.max(np.abs(_eval(xf, b, c, True) / ffine - 1.0)) for c in cand]
    c = cand[int(np.argmin(errs))]
    return {"a0": float(c[0]), "a": [float(v) for v in c[1:]], "b": [float(v) for v in b], "min_eps": float(eps),
            "power": float(p), "max_rel_err": float(min(errs)), "method": "aaa-lawson"}
