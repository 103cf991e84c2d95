"""Generates the coefficient table of the FP32 Bessel J0/J1 evaluation for
x >= 3 in qem_internal.cuh (bessel01_x2), and reports its error.

Form (the Hankel asymptotic form with fitted amplitude polynomials): with
t = x - pi/4, u = 1/x, w = u^2,
    J0(x) = x^{-1/2} (P0(w) cos t + u Q0(w) sin t)
    J1(x) = x^{-1/2} (P1(w) sin t + u Q1(w) cos t)
where P0, P1 (degree 5) and Q0, Q1 (degree 4) are near-minimax polynomial
fits on w in (0, 1/9] (Lawson-reweighted least squares on Chebyshev-spaced
points) of the exact amplitudes
    P0 = sqrt(2/pi) * sqrt(pi x / 2) (J0 cos t + Y0 sin t),
    -Q0/u = sqrt(2/pi) * sqrt(pi x / 2) (Y0 cos t - J0 sin t), and the same
for order 1 with t1 = t - pi/2, where cos t1 = sin t and sin t1 = -cos t
give +Q1/u = sqrt(2/pi) * sqrt(pi x / 2) (Y1 cos t1 - J1 sin t1), so that
J1 takes sin t and cos t of the same t.  The sqrt(2/pi) of the asymptotic
form and the signs are folded into the coefficients.  scipy.special
supplies J and Y.

    python qem4molly_b200/csrc/gen_bessel_pq.py      # prints the C table and the errors
"""
import numpy as np
from scipy import special as sp

X0 = 3.0
DEG = {"P0": 5, "Q0": 4, "P1": 5, "Q1": 4}


def amplitudes(x):
    t0 = x - np.pi / 4
    t1 = x - 3 * np.pi / 4
    a = np.sqrt(np.pi * x / 2) * np.sqrt(2 / np.pi)  # = sqrt(x)
    J0, Y0, J1, Y1 = sp.j0(x), sp.y0(x), sp.j1(x), sp.y1(x)
    P0 = a * (J0 * np.cos(t0) + Y0 * np.sin(t0))
    Q0 = -a * (Y0 * np.cos(t0) - J0 * np.sin(t0)) * x   # J0 = x^-1/2 (P0 cos t + u Q0 sin t)
    P1 = a * (J1 * np.cos(t1) + Y1 * np.sin(t1))
    Q1 = a * (Y1 * np.cos(t1) - J1 * np.sin(t1)) * x    # cos t1 = sin t, sin t1 = -cos t
    return {"P0": P0, "Q0": Q0, "P1": P1, "Q1": Q1}


def fit(w, y, deg, scale):
    """Lawson's iteration towards the minimax fit of y(w) (errors weighted by scale)."""
    V = np.vander(w, deg + 1, increasing=True)
    wt = np.ones_like(w)
    for _ in range(60):
        s = np.sqrt(wt) * scale
        c, *_ = np.linalg.lstsq(V * s[:, None], y * s, rcond=None)
        r = np.abs(V @ c - y) * scale
        wt = wt * r / np.sum(wt * r) * len(w) + 1e-300
    return c


def coefficients():
    th = np.linspace(0, np.pi, 6000)
    w = 0.5 * (1 - np.cos(th)) / X0 ** 2
    w = w[w > 0]
    x = 1 / np.sqrt(w)
    amp = amplitudes(x)
    out = {}
    for name, deg in DEG.items():
        scale = 1 / np.sqrt(x) * (1 / x if name.startswith("Q") else 1.0)  # error as it enters J
        out[name] = fit(w, amp[name], deg, scale)
    return out


def j01_fp32(x, C):
    """FP32 emulation of the device evaluation (exact sin/cos of the FP32 phase)."""
    f = np.float32
    x = x.astype(f)
    r = (1 / np.sqrt(x.astype(np.float64))).astype(f)
    u = (r * r).astype(f)
    w = (u * u).astype(f)

    def horner(c):
        acc = np.full_like(w, f(c[-1]))
        for cj in c[-2::-1]:
            acc = (acc * w + f(cj)).astype(f)
        return acc

    P0, Q0, P1, Q1 = (horner(C[n]) for n in ("P0", "Q0", "P1", "Q1"))
    t = (x - f(np.pi / 4)).astype(f)
    S, Cs = np.sin(t.astype(np.float64)).astype(f), np.cos(t.astype(np.float64)).astype(f)
    J0 = (r * (P0 * Cs + (u * Q0) * S)).astype(f)
    J1 = (r * (P1 * S + (u * Q1) * Cs)).astype(f)
    return J0.astype(np.float64), J1.astype(np.float64)


def main():
    C = coefficients()
    x = np.linspace(X0, 60.0, 200001)
    xf = x.astype(np.float32).astype(np.float64)
    J0, J1 = j01_fp32(x, C)
    e0 = np.max(np.abs(J0 - sp.j0(xf)))
    e1 = np.max(np.abs(J1 - sp.j1(xf)))
    print(f"// max |error| on [3, 60], FP32 emulation: J0 {e0:.2e}, J1 {e1:.2e}")
    for name in ("P0", "Q0", "P1", "Q1"):
        print(f"// {name}: " + ", ".join(f"{v:.9e}f" for v in C[name]))


if __name__ == "__main__":
    main()
