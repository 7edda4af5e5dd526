"""The reference's product-form factorisation dpftrf (src/C/pfcholesky.c:
52-88, with ddrsv :4-25) evaluated in extended precision (numpy longdouble,
80-bit on x86) with the reference's own sequential recurrences.  TEST
INFRASTRUCTURE ONLY: the accuracy yardstick of the product-form parity test,
never used by the product."""
import numpy as np


def dpftrf_extended(a, V):
    """(V, L, B) of dpftrf on a copy of V (n x k), in long double, rounded
    back to float64."""
    n, k = V.shape
    W = np.asarray(V, dtype=np.longdouble).copy()
    L = np.zeros((n, k), dtype=np.longdouble)
    B = np.zeros((n, k), dtype=np.longdouble)
    one = np.longdouble(1)
    for i in range(k):
        v = list(W[:, i])
        alpha = -np.longdouble(a[i])
        ll, bb = [None] * n, [None] * n
        for j in range(n):
            lj = np.sqrt(one - alpha * v[j] * v[j])
            bj = -alpha * v[j] / lj
            ll[j], bb[j] = lj, bj
            alpha = alpha + bj * bj
        L[:, i], B[:, i] = ll, bb
        for c in range(i + 1, k):
            x = list(W[:, c])
            s = np.longdouble(0)
            for r in range(n):
                x[r] = (x[r] - v[r] * s) / ll[r]
                s = s + x[r] * bb[r]
            W[:, c] = x
    return W.astype(np.float64), L.astype(np.float64), B.astype(np.float64)
