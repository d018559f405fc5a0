"""Near-minimax rational coefficients (rhmc_b200.rational.minimax_power, AAA-Lawson): the kind of
approximation the reference builds with AlgRemez (rationalapprox_calc.cc:8-177).  Checked
independently of the module's own error estimate: on a dense grid the relative error of
a0 + sum a_i/(x + b_i) against x^p is below the least-squares fit's at the same degree, the
shifts are positive (the solver needs M^dag M + b_i > 0), the numerators have the sign of the
Stieltjes representation, and up to degree 15 the error equioscillates at 2n + 2 points with
peaks within a factor 2 of each other (the minimax property)."""
import numpy as np
import pytest

from rhmc_b200 import rational as R

CASES = [(-0.5, 8, 1.41e-5), (0.25, 8, 1.41e-5), (-0.5, 15, 5.6e-6), (-0.25, 15, 5.6e-6), (0.125, 15, 5.6e-6),
         (-0.25, 20, 1.4e-6), (0.125, 20, 1.4e-6)]


def _err(c, x):
    a, b = np.array(c["a"]), np.array(c["b"])
    return (c["a0"] + (a[None, :] / (x[:, None] + b[None, :])).sum(1)) / x ** c["power"] - 1.0


def _alternants(e):
    idx = [0] + [i for i in range(1, len(e) - 1) if (e[i] - e[i - 1]) * (e[i + 1] - e[i]) <= 0] + [len(e) - 1]
    sel = []
    for i in idx:
        if sel and np.sign(e[i]) == np.sign(e[sel[-1]]):
            if abs(e[i]) > abs(e[sel[-1]]):
                sel[-1] = i
        else:
            sel.append(i)
    return sel


@pytest.mark.parametrize("p,n,eps", CASES)
def test_minimax_beats_least_squares(p, n, eps):
    mm = R.rational_power(p, n, eps)  # the default method
    assert mm.get("method") == "aaa-lawson"
    ls = R.rational_power(p, n, eps, method="lsq")
    x = np.random.default_rng(7).uniform(np.log(eps), 0.0, 100000)
    x = np.exp(np.sort(x))
    e_mm, e_ls = np.max(np.abs(_err(mm, x))), np.max(np.abs(_err(ls, x)))
    assert e_mm <= 1.01 * mm["max_rel_err"]
    assert e_mm < e_ls
    assert len(mm["b"]) == n and min(mm["b"]) > 0.0
    sgn = 1.0 if p < 0 else -1.0
    assert all(sgn * v > 0 for v in mm["a"])


@pytest.mark.parametrize("p,n,eps", CASES[:5])
def test_minimax_equioscillates(p, n, eps):
    c = R.minimax_power(p, n, eps)
    e = _err(c, np.geomspace(eps, 1.0, 200000))
    peaks = np.abs(e[_alternants(e)])
    assert len(peaks) >= 2 * n + 1
    assert peaks.max() / np.median(peaks) < 2.0


def test_minimax_rejects_bad_powers():
    with pytest.raises(ValueError):
        R.minimax_power(1.5, 8, 1e-4)
    with pytest.raises(ValueError):
        R.rational_power(-0.5, 8, 1e-4, method="remez")
