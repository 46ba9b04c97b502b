"""Dense-matrix helpers for the known-answer tests: `DenseCsc` of the
reference's tests (src/solver/tests.zig), which drops exact zeros."""
import numpy as np


def dense_csc(a):
    a = np.asarray(a, dtype=np.float64)
    n = a.shape[0]
    cp = [0]
    ri = []
    vals = []
    for j in range(n):
        for i in range(n):
            if a[i, j] != 0:
                ri.append(i)
                vals.append(a[i, j])
        cp.append(len(ri))
    return np.array(cp, np.uint32), np.array(ri, np.uint32), np.array(vals)


def is_perm(q, n):
    return len(q) == n and sorted(int(v) for v in q) == list(range(n))


def random_pattern(rng, n, density, full_diag=True):
    cols = []
    for j in range(n):
        cols.append([i for i in range(n) if (i == j and full_diag) or rng.random() < density])
    cp = np.cumsum([0] + [len(c) for c in cols]).astype(np.uint32)
    ri = np.array([r for c in cols for r in c], dtype=np.uint32)
    return cp, ri
