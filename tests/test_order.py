"""Column ordering (BTF + AMD), oracle and product, against the reference's
known-answer structures (src/solver/tests.zig:2600-2800) and properties
(src/solver/order.zig:721-827, tests.zig:2809-2895)."""
import numpy as np
import pytest

from egspice_b200 import symbolic
from tests.dense import dense_csc, is_perm, random_pattern

STAR = [[1, 1, 1, 1, 1], [1, 1, 0, 0, 0], [1, 0, 1, 0, 0], [1, 0, 0, 1, 0], [1, 0, 0, 0, 1]]
BTF = [[1, 1, 1, 0], [1, 1, 0, 0], [0, 0, 1, 1], [0, 0, 1, 1]]


def both(oracle, cp, ri):
    q1 = oracle.order(cp, ri)
    q2 = symbolic.order(cp, ri)
    assert q1 is not None and q2 is not None
    assert np.array_equal(q1, q2), "product order differs from the oracle's"
    return q1


def test_star_defers_hub(oracle):
    cp, ri, _ = dense_csc(STAR)
    q = both(oracle, cp, ri)
    assert is_perm(q, 5)
    assert q[3] == 0 or q[4] == 0
    qa = oracle.amd(cp, ri)
    assert qa[3] == 0 or qa[4] == 0


def test_btf_sink_block_first(oracle):
    cp, ri, _ = dense_csc(BTF)
    q = both(oracle, cp, ri)
    assert q[0] < 2 and q[1] < 2 and q[2] >= 2 and q[3] >= 2


def test_btf_three_blocks_topological(oracle):
    cp, ri, _ = dense_csc([[1, 1, 1], [0, 1, 1], [0, 0, 1]])
    assert list(both(oracle, cp, ri)) == [0, 1, 2]


def test_chain_identity_k4(oracle):
    a = np.eye(6) + np.eye(6, k=1) + np.eye(6, k=-1)
    cp, ri, _ = dense_csc(a)
    assert is_perm(oracle.amd(cp, ri), 6)
    cp, ri, _ = dense_csc(np.eye(3))
    assert is_perm(both(oracle, cp, ri), 3)
    cp, ri, _ = dense_csc(np.ones((4, 4)))
    assert is_perm(oracle.amd(cp, ri), 4)


def test_empty_and_one(oracle):
    assert len(oracle.order(np.array([0], np.uint32), np.zeros(0, np.uint32))) == 0
    assert list(both(oracle, np.array([0, 1], np.uint32), np.array([0], np.uint32))) == [0]


def test_arrowhead_hub_last(oracle):
    n = 8
    a = np.eye(n)
    a[0, :] = 1
    a[:, 0] = 1
    cp, ri, _ = dense_csc(a)
    qa = oracle.amd(cp, ri)
    assert qa[n - 1] == 0 or qa[n - 2] == 0
    # order -> factor: the hub is not factored first (tests.zig:2895-2922)
    cp, ri, vals = dense_csc([[5, 1, 1, 1], [1, 2, 0, 0], [1, 0, 3, 0], [1, 0, 0, 4]])
    q = both(oracle, cp, ri)
    assert q[0] != 0
    lu = oracle.SparseLu(cp, ri, q)
    assert lu.factor(vals) == 0
    x = lu.solve([8, 3, 4, 5])
    a = np.array([[5, 1, 1, 1], [1, 2, 0, 0], [1, 0, 3, 0], [1, 0, 0, 4]], float)
    assert np.allclose(a @ x, [8, 3, 4, 5], rtol=1e-13)


def test_random_patterns_are_permutations(oracle):
    rng = np.random.default_rng(0x0DE7)
    for t in range(300):
        n = t + 1 if t < 64 else int(rng.integers(1, 65))
        dens = 0.3 + 0.6 * rng.random() if t % 4 == 0 else 0.05 * rng.random()
        cp, ri = random_pattern(rng, n, dens)
        q = both(oracle, cp, ri)
        assert is_perm(q, n)
        assert is_perm(oracle.amd(cp, ri), n)


def test_short_slabs_fail_cleanly_or_agree(oracle):
    rng = np.random.default_rng(0x0DE8)
    n = 24
    cp, ri = random_pattern(rng, n, 0.2)
    full = oracle.ws_size(n, int(cp[-1]))
    want = oracle.order(cp, ri, slab_len=full)
    want_amd = oracle.amd(cp, ri, slab_len=full)
    passed = 0
    for ln in range(0, full + 1, 7):
        q = oracle.order(cp, ri, slab_len=ln)
        if q is not None:
            assert np.array_equal(q, want)
            passed += 1
        qa = oracle.amd(cp, ri, slab_len=ln)
        if qa is not None:
            assert np.array_equal(qa, want_amd)
    assert passed > 0


def test_chol_count_cap(oracle):
    rng = np.random.default_rng(0x0DE9)
    n = 40
    for _ in range(50):
        cp, ri = random_pattern(rng, n, 0.08)
        perm = rng.permutation(n).astype(np.uint32)
        full = oracle.chol_count(cp, ri, perm)
        for cap in (n, full - 1, full, full + 1):
            got = oracle.chol_count(cp, ri, perm, cap)
            if full < cap:
                assert got == full
            else:
                assert got >= cap


def test_degree10_patterns_fit_workspace(oracle):
    rng = np.random.default_rng(0x46)
    for n in (2000, 4000):
        cols = []
        for j in range(n):
            s = {j}
            for _ in range(10):
                s.add(int(rng.integers(0, n)))
            cols.append(sorted(s))
        cp = np.cumsum([0] + [len(c) for c in cols]).astype(np.uint32)
        ri = np.array([r for c in cols for r in c], np.uint32)
        q = both(oracle, cp, ri)
        assert is_perm(q, n)


def test_rail_last_chains_never_fill_more_than_natural(oracle):
    rng = np.random.default_rng(42)
    for _ in range(300):
        n = int(rng.integers(6, 41))
        m = n - int(rng.integers(1, 4))
        d = np.zeros((n, n), bool)
        for i in range(1, m):
            d[i, i - 1] = d[i - 1, i] = True
            if rng.random() < 0.3 and i >= 2:
                d[i, i - 2] = d[i - 2, i] = True
        for rl in range(m, n):
            for i in range(m):
                if rng.random() < 0.7:
                    d[rl, i] = d[i, rl] = True
        a = np.where(d, -1.0, 0.0)
        np.fill_diagonal(a, 2 * n)
        cp, ri, vals = dense_csc(a)
        q = both(oracle, cp, ri)

        def fill(order):
            lu = oracle.SparseLu(cp, ri, order)
            assert lu.factor(vals) == 0
            t = lu.tape()
            return len(t["li"]) + len(t["ui"])

        assert fill(q) <= fill(np.arange(n, dtype=np.uint32))


@pytest.mark.parametrize("make", ["chain", "opamp", "ring", "ladder", "grid"])
def test_config_patterns_bit_exact(oracle, make):
    from egspice_b200 import decks
    net = {
        "chain": lambda: decks.inverter_chain(2),
        "opamp": lambda: decks.miller_opamp(2),
        "ring": lambda: decks.ring_oscillator(2, stages=63),
        "ladder": lambda: decks.rc_diode_ladder(5000, 2, seed=9),
        "grid": lambda: decks.power_grid(2, side=40, loads=20),
    }[make]()
    q = both(oracle, net.col_ptr, net.row_idx)
    assert is_perm(q, net.n)
