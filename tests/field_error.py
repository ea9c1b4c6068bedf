"""The stated error model of the FP32-compensated field, for tests.

Band pairs (|d| <= 16 eps) are summed in FP64, so what remains is the far
pairs' FP32 arithmetic on terms of size eps^2/d^2: about 1e-9 of the band-charge
scale ||S||, S_i^2 = sum over target i's band of (q_j/2)^2.  The bound a test
asserts is therefore 1e-6 of ||E||, or 2e-9 of ||S|| where the field is that
small (a Landau field near a node of its oscillation)."""
import numpy as np

BAND = 16.0


def band_charge_scale(xs, q, L, eps):
    """||S||: sqrt of the sum over targets of the sum of (q_j/2)^2 over each
    target's band |x_i - x_j| <= 16 eps (periodic)."""
    xw = np.mod(np.asarray(xs, dtype=np.float64), L)
    o = np.argsort(xw, kind="stable")
    xs_ = xw[o]
    q2 = (0.5 * np.asarray(q, dtype=np.float64)[o]) ** 2
    X = np.concatenate([xs_ - L, xs_, xs_ + L])
    P = np.concatenate([[0.0], np.cumsum(np.concatenate([q2, q2, q2]))])
    lo = np.searchsorted(X, xw - BAND * eps, "left")
    hi = np.searchsorted(X, xw + BAND * eps, "right")
    return float(np.sqrt(np.sum(P[hi] - P[lo])))


def fp32c_bound(xs, q, L, eps, e_ref):
    """Largest ||E - E_ref|| the FP32-compensated field is allowed."""
    return max(1e-6 * float(np.linalg.norm(e_ref)), 2e-9 * band_charge_scale(xs, q, L, eps))
