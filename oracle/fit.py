"""Test infrastructure only: the reference's ISF analysis restated for checking the engine's
on-device fits (ddm_fit_isf). The reference does this step in Python
(resources/python_tools/plot_averaged.py) with scipy.optimize.curve_fit, which is
MINPACK's Levenberg-Marquardt (lmdif); this module calls the same scipy routine with the
script's model and starting point, so the oracle is the reference's own method. The scipy
version of this environment is recorded by the tests that use it (scipy.__version__).

Nothing in the engine imports this module.
"""
from __future__ import annotations

import numpy as np
import scipy
import scipy.optimize as opt

P0 = (6.0, 3e-2, 4e-3)  # plot_averaged.py:77: (F, A, B)


def fit_func(x, F, A, B):
    """plot_averaged.py:57-58 (the where= guard keeps exp's argument below 700)."""
    return A * (1 - np.exp(np.minimum(-x * F, 700.0))) + B


def start_from_data(tau, isf):
    """The engine's data-read start (DDM_FIT_START_DATA): B = first value, A = largest rise
    above it, F = ln 2 / first lag whose value reaches half the rise."""
    tau = np.asarray(tau, float)
    y = np.asarray(isf, float)
    b = y[0]
    a = y.max() - b
    if not a > 0:
        a = max(abs(b), 1e-300)
    hit = np.nonzero(y >= b + 0.5 * a)[0]
    t_half = tau[hit[0]] if hit.size else tau[-1]
    return (np.log(2.0) / max(t_half, 1e-300), a, b)


def fit_curve(tau, isf, tight: bool = True, start: str = "data"):
    """(F, A, B), (sigma_F, sigma_A, sigma_B) as plot_averaged.py:64-90 computes them, from
    the script's p0 (start="script") or the data-read start. With tight=True the solver runs
    to its tolerance floor (the exact least-squares minimum the engine's solver also converges
    to); tight=False uses curve_fit's defaults, as the script."""
    kw = dict(ftol=1e-15, xtol=1e-15, gtol=1e-15, maxfev=200000) if tight else {}
    p0 = P0 if start == "script" else start_from_data(tau, isf)
    popt, pcov = opt.curve_fit(fit_func, np.asarray(tau, float), np.asarray(isf, float), p0=p0, **kw)
    return popt, np.sqrt(np.diag(pcov))


def diffusion(F, q):
    """plot_averaged.py:93-141: ln F = 2 ln q + c over F > 0, D = exp(c), sigma_D = sigma_c D."""
    F = np.asarray(F, float)
    q = np.asarray(q, float)
    keep = (F > 0) & np.isfinite(F)
    lnF, lnq = np.log(F[keep]), np.log(q[keep])
    popt, pcov = opt.curve_fit(lambda x, c: 2 * x + c, xdata=lnq, ydata=lnF)
    c, c_err = popt[0], np.sqrt(pcov[0, 0])
    return np.exp(c), c_err * np.exp(c)


def q_vector(lambdas, um_per_px: float = 1.0):
    """plot_averaged.py:258-261: q = 2 pi / lambda, lambda in micrometres."""
    return 2 * np.pi / (np.asarray(lambdas, float) * um_per_px)


SCIPY_VERSION = scipy.__version__
