"""The transposed TRT collision used by the adjoint kernel (k_adj_bulk,
trt_adjoint in csrc/bfx_adjoint.cu), restated here in numpy with the kernel's
pairwise arrangement, against central finite differences of the TRT
collision (BF.metal:3063-3093) in FP64.  CPU only."""
from __future__ import annotations

import numpy as np

C = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1], [1, 0, -1], [-1, 0, 1],
              [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]], dtype=np.float64)
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17])


def feq(rho, u):
    cu = C @ u
    return W * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (u @ u))


def trt(f, wp, wm):
    rho = f.sum()
    u = (f @ C) / rho
    e = feq(rho, u)
    fp, fm = 0.5 * (f + f[OPP]), 0.5 * (f - f[OPP])
    ep, em = 0.5 * (e + e[OPP]), 0.5 * (e - e[OPP])
    return f - wp * (fp - ep) - wm * (fm - em)


def trt_adjoint(lam, u, wp, wm):
    """Pairwise form of the kernel: mu_j = lam_j - Lam_j + A + B . (c_j - u)."""
    u2 = u @ u
    L = np.zeros(19)
    L[0] = wp * lam[0]
    A = L[0] * W[0] * (1 - 1.5 * u2)
    B = L[0] * W[0] * (-3 * u)
    for q in range(1, 19, 2):
        lp, lm = 0.5 * (lam[q] + lam[q + 1]), 0.5 * (lam[q] - lam[q + 1])
        Lq, Lo = wp * lp + wm * lm, wp * lp - wm * lm
        L[q], L[q + 1] = Lq, Lo
        cu = C[q] @ u
        even = 1 + 4.5 * cu * cu - 1.5 * u2
        S, D = Lq + Lo, Lq - Lo
        A += W[q] * (S * even + D * 3 * cu)
        B += W[q] * (C[q] * (3 * D + 9 * cu * S) - 3 * u * S)
    return lam - L + (A - B @ u) + C @ B


def test_transposed_trt_matches_finite_differences():
    rng = np.random.default_rng(7)
    for wp, wm in ((1.9, 1.2), (1.05, 0.8), (1.6, 1.6)):
        u = rng.uniform(-0.08, 0.08, 3)
        f = feq(1.0 + rng.uniform(-0.05, 0.05), u) * (1 + 0.02 * rng.standard_normal(19))
        lam = rng.standard_normal(19)
        rho = f.sum()
        mu = trt_adjoint(lam, (f @ C) / rho, wp, wm)
        h = 1e-6
        fd = np.empty(19)
        for j in range(19):
            e = np.zeros(19)
            e[j] = h
            fd[j] = lam @ (trt(f + e, wp, wm) - trt(f - e, wp, wm)) / (2 * h)
        assert np.max(np.abs(mu - fd)) < 1e-8 * max(1.0, np.max(np.abs(fd)))


def test_equilibrium_velocity_adjoint_matches_finite_differences():
    """d equilibrium_q(1, u) / du_b = w_q (3 c_qb + 9 (c_q.u) c_qb - 3 u_b) (k_adj_rare)."""
    rng = np.random.default_rng(3)
    u = rng.uniform(-0.1, 0.1, 3)
    lam = rng.standard_normal(19)
    G = np.array([np.sum(lam * W * (3 * C[:, b] + 9 * (C @ u) * C[:, b] - 3 * u[b])) for b in range(3)])
    h = 1e-6
    fd = np.array([lam @ (feq(1.0, u + h * np.eye(3)[b]) - feq(1.0, u - h * np.eye(3)[b])) / (2 * h) for b in range(3)])
    assert np.allclose(G, fd, atol=1e-9)
    # the refill momentum sum_q feq_q(1, u) c_q has the identity as its velocity derivative
    J = np.array([(feq(1.0, u + h * np.eye(3)[b]) @ C - feq(1.0, u - h * np.eye(3)[b]) @ C) / (2 * h) for b in range(3)])
    assert np.allclose(J, np.eye(3), atol=1e-8)
