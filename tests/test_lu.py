"""Sparse LU (oracle and product tape) against the reference's known
answers (src/solver/tests.zig:2923-3380, src/solver/sparse_lu.zig:1450-1745)."""
import numpy as np

from egspice_b200 import decks, symbolic
from tests.dense import dense_csc, random_pattern

BSIMSOI_BODY = [[2.0e-20, -1.0e-20, -1.0e-20, 0.0], [-1.0e-6, 1.0e3, -9.0e-4, 1.0e-3],
                [1.0e-6, -9.0e-4, 2.0e-3, -1.0e-3], [0.0, 0.0, -1.0e-3, 1.0]]


def ident(n):
    return np.arange(n, dtype=np.uint32)


def test_mna_zero_diagonal(oracle):
    a = [[1e-3, 0, 1], [0, 2e-3, -1], [1, -1, 0]]
    cp, ri, v = dense_csc(a)
    lu = oracle.SparseLu(cp, ri, ident(3))
    assert lu.factor(v) == 0
    x = lu.solve([0, 0, 5])
    assert np.allclose(np.array(a) @ x, [0, 0, 5], atol=1e-12)


def test_row_scaled_pivot_keeps_floating_body(oracle):
    a = np.array(BSIMSOI_BODY)
    xt = np.array([0.03526, 0.9, 0.1, 1.1])
    b = a @ xt
    cp, ri, v = dense_csc(a)
    lu = oracle.SparseLu(cp, ri, ident(4))
    assert lu.factor(v) == 0
    t = lu.tape()
    assert t["pinv"][0] == 0 and t["scaled_pivot"][0] == 1
    assert np.allclose(lu.solve(b), xt, rtol=1e-9)
    assert lu.refactor(v, 1e-12) == 0
    assert np.allclose(lu.solve(b), xt, rtol=1e-9)
    pt = symbolic.tape(cp, ri, v, ident(4))
    assert np.array_equal(pt["pinv"], t["pinv"]) and pt["flags"][0] & 2


def test_void_unknown_unit_pivot(oracle):
    cp = np.array([0, 3, 6, 9], np.uint32)
    ri = np.array([0, 1, 2, 0, 1, 2, 0, 1, 2], np.uint32)
    v = np.array([2, 0, 1, 0, 0, 0, 1, 0, 3], float)
    lu = oracle.SparseLu(cp, ri, ident(3))
    assert lu.factor(v) == 0
    assert lu.tape()["void_col"][1] == 1
    assert np.allclose(lu.solve([5, 0, 7]), [8 / 5, 0, 9 / 5], atol=1e-12)
    assert lu.refactor([4, 0, 1, 0, 0, 0, 1, 0, 5], 0) == 0
    assert np.allclose(lu.solve([5, 0, 7]), [18 / 19, 0, 23 / 19], atol=1e-12)
    pt = symbolic.tape(cp, ri, v, ident(3))
    assert pt["flags"][1] & 1 and len(pt["void_slots"]) == len(lu.tape()["void_slots"])


def test_fabricated_pivot_activation_is_rejected(oracle):
    cp = np.array([0, 2, 4], np.uint32)
    ri = np.array([0, 1, 0, 1], np.uint32)
    for q in ([0, 1], [1, 0]):
        for vals in ([2, 0, 0, 4], [2, 1, 0, 0], [2, 0, 1, 0], [2, 1, 1, 0]):
            lu = oracle.SparseLu(cp, ri, q)
            assert lu.factor([2, 0, 0, 0]) == 0
            assert lu.refactor(vals, 1e-12) != 0


def test_singular_rejected(oracle):
    cp, ri, v = dense_csc([[1, 1], [1, 1]])
    assert oracle.SparseLu(cp, ri, ident(2)).factor(v) != 0
    assert symbolic.tape(cp, ri, v, ident(2)) is None


def test_offdiagonal_pivot_hands_off_its_diagonal(oracle):
    a = [[1e-9, 1, 0], [1, 1e-9, 0], [0, 5, 1]]
    cp, ri, v = dense_csc(a)
    lu = oracle.SparseLu(cp, ri, ident(3))
    assert lu.factor(v) == 0
    assert list(lu.tape()["pinv"]) == [1, 0, 2]
    assert list(symbolic.tape(cp, ri, v, ident(3))["pinv"]) == [1, 0, 2]
    assert np.allclose(np.array(a) @ lu.solve([1, 2, 3]), [1, 2, 3], rtol=1e-12)


def test_repivot_past_fill_cap_keeps_previous_pivots(oracle):
    a = np.array([[2, -1, 0, 0], [-1, 2, -1, 0], [0, -1, 2, -1], [0, 0, -1, 2]], float)
    cp, ri, v = dense_csc(a)
    capped = oracle.SparseLu(cp, ri, ident(4), fill_cap=1.0)
    free = oracle.SparseLu(cp, ri, ident(4))
    assert capped.factor(v) == 0 and free.factor(v) == 0
    base = len(capped.tape()["li"]) + len(capped.tape()["ui"])
    a[0, 0] = 1e-5
    cp, ri, v = dense_csc(a)
    assert free.factor(v) == 0
    assert len(free.tape()["li"]) + len(free.tape()["ui"]) > base
    assert capped.factor(v) == 0
    t = capped.tape()
    assert len(t["li"]) + len(t["ui"]) == base and list(t["pinv"]) == [0, 1, 2, 3]


def test_overflow_fails_factor_and_replay(oracle):
    cp = np.array([0, 2, 3, 6], np.uint32)
    ri = np.array([0, 1, 1, 0, 1, 2], np.uint32)
    q = np.array([0, 1, 2], np.uint32)
    benign = np.ones(6)
    over = np.array([1, 1, 1, 1.5e308, -1.5e308, 1])
    assert oracle.SparseLu(cp, ri, q).factor(over) != 0
    lu = oracle.SparseLu(cp, ri, q)
    assert lu.factor(benign) == 0
    assert lu.refactor(over, 1e-12) != 0
    assert lu.refactor(over, 0) != 0
    assert lu.refactor(benign, 1e-12) == 0


def test_random_systems_scaled_residual_and_replay_bitwise(oracle):
    """sparse_lu.zig TestSystem: diagonal pushed past its column sum, 15 %
    zero diagonals (MNA branch rows); factor, refactor and both solves
    leave a small scaled residual, and product tapes equal the oracle's."""
    rng = np.random.default_rng(0x1A7E5)
    for trial in range(80):
        n = 2 + trial % 40
        cp, ri = random_pattern(rng, n, 0.3)
        v = rng.uniform(-1, 1, len(ri))
        for j in range(n):
            rows = ri[cp[j]:cp[j + 1]]
            dpos = cp[j] + int(np.nonzero(rows == j)[0][0])
            s = np.abs(v[cp[j]:cp[j + 1]]).sum() - abs(v[dpos])
            v[dpos] = 0.0 if (s > 0 and rng.random() < 0.15) else v[dpos] + np.copysign(s, v[dpos])
        q = oracle.order(cp, ri)
        lu = oracle.SparseLu(cp, ri, q)
        if lu.factor(v) != 0:
            continue
        a = np.zeros((n, n))
        for j in range(n):
            a[ri[cp[j]:cp[j + 1]], j] = v[cp[j]:cp[j + 1]]
        b = rng.uniform(-1, 1, n)
        for x, mat in ((lu.solve(b), a), (lu.solve_t(b), a.T)):
            r = np.abs(mat @ x - b).max() / (n * np.abs(a).max() * np.abs(x).max() * n * 2.2e-16)
            assert r < 100
        t1 = lu.tape()
        pt = symbolic.tape(cp, ri, v, q)
        for k in ("pinv", "lp", "li", "up", "ui", "prow"):
            assert np.array_equal(pt[k], t1[k]), k
        assert np.array_equal(pt["lx"].view(np.uint64), t1["lx"].view(np.uint64))
        v2 = v * rng.uniform(0.95, 1.05, len(v))
        x_before = lu.solve(b)
        if lu.refactor(v2, 1e-12) == 0:
            fresh = oracle.SparseLu(cp, ri, q)
            assert fresh.factor(v2) == 0


def test_supernodal_walk_on_a_mesh(oracle):
    """A mesh's factor takes the supernodal DFS (panels hold most of L,
    sparse_lu.zig:754-910); the product tape equals the oracle's there too."""
    net = decks.power_grid(1, side=30, loads=5)
    from oracle.pyoracle import op_lanes  # noqa: F401  (imports the oracle)
    cp, ri = net.col_ptr, net.row_idx
    rng = np.random.default_rng(7)
    v = np.zeros(net.nnz)
    for j in range(net.n):
        for p in range(cp[j], cp[j + 1]):
            v[p] = 4.0 if ri[p] == j else -rng.uniform(0.5, 1.0)
    q = oracle.order(cp, ri)
    lu = oracle.SparseLu(cp, ri, q)
    assert lu.factor(v) == 0
    t = lu.tape()
    pt = symbolic.tape(cp, ri, v, q)
    for k in ("pinv", "lp", "li", "up", "ui"):
        assert np.array_equal(pt[k], t[k]), k
    assert t["n_panels"] > 0
