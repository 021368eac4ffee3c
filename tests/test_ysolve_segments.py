"""The y-solve's segment split on the CPU: each mode's NM rows cut into P
segments of Le = ceil(NM / P) rows (the last ones shorter or empty), both
Thomas recurrences run per segment from a zero start with the product of
the multipliers, the segments' affine maps composed in order (forward) and
in reverse (backward), and a second pass adding product x entering value --
the scheme of k_thomas_tile_scan -- against the serial sweeps with the same
inverse pivots, for every NM the tiles serve (1 to 256) and P = 16."""
import numpy as np
import pytest


def pivots(dd, dl, du, lam):
    piv = np.zeros(len(dd))
    for b in range(len(dd)):
        d = dd[b] + lam
        if b > 0:
            d = d - dl[b] * piv[b - 1] * du[b - 1]
        piv[b] = 1.0 / d
    return piv


def serial(piv, dl, du, r):
    NM = len(r)
    g = np.zeros(NM, complex)
    x = np.zeros(NM, complex)
    for b in range(NM):
        g[b] = r[b] - (dl[b] * piv[b - 1] * g[b - 1] if b > 0 else 0)
    for b in range(NM - 1, -1, -1):
        x[b] = g[b] * piv[b] if b == NM - 1 else (g[b] - du[b] * x[b + 1]) * piv[b]
    return x


def segments(piv, dl, du, r, P):
    NM = len(r)
    Le = (NM + P - 1) // P
    c = np.array(r, complex)
    A = np.ones(P)
    C = np.zeros(P, complex)
    for kk in range(P):  # forward, from g = 0 at each segment's start
        s0, nr = kk * Le, max(0, min(Le, NM - kk * Le))
        g, h = 0j, 1.0
        for u in range(nr):
            b = s0 + u
            w = dl[b] * piv[b - 1] if b > 0 else 0.0
            g = c[b] - w * g
            h = -w * h
            c[b] = g
        if nr:
            A[kk], C[kk] = h, g
    for kk in range(P):  # entering value: the maps before, composed in order
        s0, nr = kk * Le, max(0, min(Le, NM - kk * Le))
        gi = 0j
        for q in range(kk):
            gi = C[q] + A[q] * gi
        h = 1.0
        for u in range(nr):
            b = s0 + u
            w = dl[b] * piv[b - 1] if b > 0 else 0.0
            h = -w * h
            c[b] = c[b] + h * gi
    A[:] = 1.0
    C[:] = 0j
    for kk in range(P):  # backward, from x = 0 above each segment
        s0, nr = kk * Le, max(0, min(Le, NM - kk * Le))
        x, k = 0j, 1.0
        for u in range(nr - 1, -1, -1):
            b = s0 + u
            if b == NM - 1:
                x, beta = c[b] * piv[b], 0.0
            else:
                x, beta = (c[b] - du[b] * x) * piv[b], -du[b] * piv[b]
            k = beta * k
            c[b] = x
        if nr:
            A[kk], C[kk] = k, x
    for kk in range(P):  # the value above: the maps after, composed from the top
        s0, nr = kk * Le, max(0, min(Le, NM - kk * Le))
        xi = 0j
        for q in range(P - 1, kk, -1):
            xi = C[q] + A[q] * xi
        k = 1.0
        for u in range(nr - 1, -1, -1):
            b = s0 + u
            beta = 0.0 if b == NM - 1 else -du[b] * piv[b]
            k = beta * k
            c[b] = c[b] + k * xi
    return c


@pytest.mark.parametrize("NM", [1, 2, 3, 8, 15, 16, 17, 31, 64, 100, 127, 128, 129, 200, 255, 256])
def test_segment_join_equals_serial_sweeps(NM):
    rng = np.random.default_rng(NM)
    # a y-operator of the solver's kind: negative diagonal, positive couplings
    dl = rng.uniform(0.2, 1.0, NM)
    du = rng.uniform(0.2, 1.0, NM)
    dd = -(dl + du) - rng.uniform(0.0, 0.1, NM)
    for lam in (-1e-3, -0.5, -40.0):  # small, moderate and large kx^2 + kz^2
        piv = pivots(dd, dl, du, lam)
        r = rng.standard_normal(NM) + 1j * rng.standard_normal(NM)
        ref = serial(piv, dl, du, r)
        got = segments(piv, dl, du, r, 16)
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
