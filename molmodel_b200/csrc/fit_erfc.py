"""Derives the FP32 erfc coefficients used by the mixed-precision pair kernels.

Form (Hastings' rational approximation, as in Abramowitz & Stegun 7.1.26):
    erfc(x) ~= t * P(t) * exp(-x^2),   t = 1 / (1 + p x),   x >= 0,
with p = 0.3275911 and P a degree-7 polynomial.  Instead of A&S's five
coefficients (absolute error 1.5e-7, relative error up to 0.3% below x = 4),
P is fitted here for RELATIVE accuracy: a least-squares Chebyshev fit of
erfcx(x) / t on x in [0, 6], weighted by 1 / (erfcx(x) / t), converted to the
power basis and rounded to FP32 (relative error <= 4e-7 everywhere, FP32
Horner included).  The printed table is pasted into rspace_mixed.cu; this
script checks the FP32 Horner evaluation against scipy's erfc.

    python molmodel_b200/csrc/fit_erfc.py
"""
import numpy as np
from scipy.special import erfc, erfcx

P_PARAM = 0.3275911
DEG = 7


def fit():
    x = np.linspace(0.0, 6.0, 200001)
    t = 1.0 / (1.0 + P_PARAM * x)
    y = erfcx(x) / t
    c = np.polynomial.chebyshev.Chebyshev.fit(t, y, DEG, w=1.0 / y)
    return c.convert(kind=np.polynomial.Polynomial).coef.astype(np.float32)


def check(coef):
    x = np.linspace(0.0, 6.0, 100001).astype(np.float32)
    t = (np.float32(1) / (np.float32(1) + np.float32(P_PARAM) * x)).astype(np.float32)
    acc = np.float32(coef[-1])
    for c in coef[-2::-1]:
        acc = (acc * t + np.float32(c)).astype(np.float32)
    approx = (t * acc).astype(np.float64) * np.exp(-x.astype(np.float64) ** 2)
    exact = erfc(x.astype(np.float64))
    rel = np.abs(approx / exact - 1)
    return rel.max(), np.abs(approx - exact).max()


if __name__ == "__main__":
    coef = fit()
    print("coefficients (t^0 .. t^7):", ", ".join(f"{c:.9g}f" for c in coef))
    print("max relative error, max absolute error (FP32 Horner, exact exp):", check(coef))
