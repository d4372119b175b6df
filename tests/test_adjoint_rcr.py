"""Hand derivatives of the RCR implicit coefficients against central
differences (CPU; the adjoint's 0D coupling part)."""
import numpy as np

from crimsonflowsolver_b200.adjoint import rcr_coeffs
from oracle import pyoracle as po


def test_rcr_coeffs_match_oracle():
    for args in [(100.0, 1e-4, 1000.0, 0.0, 5.0, 2.0, 1e-3), (80.0, 2e-4, 1200.0, 3.0, -1.0, 0.5, 5e-4)]:
        Rp, C, Rd, Pd, Pn, Qn, tau = args
        s, o = po.rcr_coeffs(Rp, C, Rd, Pd, Pd, Pn, Qn, tau)
        s2, o2 = rcr_coeffs(*args)[:2]
        assert abs(s2 - s) <= 1e-13 * abs(s)
        assert abs(o2 - o) <= 1e-13 * max(abs(o), 1.0)


def test_rcr_partials_vs_central_differences():
    base = np.array([100.0, 1e-4, 1000.0, 0.5, 7.0, 3.0])   # Rp, C, Rd, Pd, Pn, Qn
    tau = 1e-3
    s, o, ds, do, doP, doQ = rcr_coeffs(*base, tau)
    an_s = np.array([ds[0], ds[1], ds[2]])
    an_o = np.array([do[0], do[1], do[2], doP, doQ])
    idx_s = [0, 1, 2]
    idx_o = [0, 1, 2, 4, 5]
    for k, i in enumerate(idx_s):
        h = 1e-6 * abs(base[i])
        p, m = base.copy(), base.copy()
        p[i] += h
        m[i] -= h
        fd = (rcr_coeffs(*p, tau)[0] - rcr_coeffs(*m, tau)[0]) / (2 * h)
        assert abs(fd - an_s[k]) <= 1e-6 * max(abs(fd), 1e-12), (i, fd, an_s[k])
    for k, i in enumerate(idx_o):
        h = 1e-6 * abs(base[i])
        p, m = base.copy(), base.copy()
        p[i] += h
        m[i] -= h
        fd = (rcr_coeffs(*p, tau)[1] - rcr_coeffs(*m, tau)[1]) / (2 * h)
        assert abs(fd - an_o[k]) <= 1e-6 * max(abs(fd), 1e-12), (i, fd, an_o[k])
