"""Test infrastructure: numpy restatement of the reference's Tab
(sun.cpp:580-670) and FourierTrafo (sun.cpp:365-411) in the form the GPU
kernels compute them (clover sum of plane a < b, F_ab = (C_ab - C_ab^dag)/8,
the per-site trace sums e_j, t_ab, g_b), checked against the reference's own
routines in tests/test_tab.py."""
import numpy as np


def tr2(a):
    return float(np.real(np.trace(a @ a)))


def clover(u, O, i, a, b):
    """C_ab at site i: the four leaves of sun.cpp:603-616."""
    H = lambda m: np.conj(m.T)  # noqa: E731
    right, up = O.getplus(i, a), O.getplus(i, b)
    left, down = O.getminus(i, a), O.getminus(i, b)
    downright, downleft, upleft = O.getplus(down, a), O.getminus(down, a), O.getminus(up, a)
    U = lambda s, d: u[s, d]  # noqa: E731
    return (U(i, a) @ U(right, b) @ H(U(up, a)) @ H(U(i, b))
            + U(i, b) @ H(U(upleft, a)) @ H(U(left, b)) @ U(left, a)
            + H(U(left, a)) @ H(U(downleft, b)) @ U(downleft, a) @ U(down, b)
            + H(U(down, b)) @ U(down, a) @ U(downright, b) @ H(U(i, a)))


def tab_site(u, pi, Pi, O, i, npt):
    D = O.dim
    pp = [pi[i, j] + Pi[i, j] for j in range(D)]
    e = [tr2(p) for p in pp]
    t = np.zeros((D, D))
    g = np.zeros(D)
    for a in range(D):
        for b in range(a + 1, D):
            C = clover(u, O, i, a, b)
            F = (C - np.conj(C.T)) / 8
            t[a, b] = t[b, a] = tr2(F)
            if a == 0:
                g[b] = -float(np.imag(np.trace(pp[b] @ F)))
    tsum = sum(t[a, b] for a in range(D) for b in range(a + 1, D))
    m = np.zeros(npt)
    m[0] = 0.25 * sum(e) - tsum
    m[1] = g.sum()
    for k in range(npt - 2):
        m[2 + k] = -0.5 * e[k] + 0.25 * sum(e) - 2.0 * t[:, k].sum() + tsum
    return m


def fourier(u, O, nc):
    n = O.dims[0]
    z = np.zeros(n)
    for i in range(n):
        for a in range(O.dim):
            for b in range(a + 1, O.dim):
                P = u[i, a] @ u[O.getplus(i, a), b] @ np.conj(u[O.getplus(i, b), a].T) @ np.conj(u[i, b].T)
                z[i] += 1.0 - np.real(np.trace(P)) / nc
    return np.abs(np.fft.ifft(z))
