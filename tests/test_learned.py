"""The learned warm start on the GPU (include/espice_learned.h): the
tensor-core forward and backward against the CPU oracle (oracle/mlp.py,
which rounds the GEMM operands to BF16 where the GPU does), training, and
what the trained network gains on a Monte-Carlo op-amp operating-point
sweep: fewer Newton iterations from its start points than from the nominal
operating point, converged by the same Newton to the same tolerance."""
import numpy as np
import pytest

from egspice_b200 import abi, decks
from egspice_b200.lanes import Lanes
from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _data(n, d, o, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, d)) * rng.uniform(0.5, 2.0, size=d) + rng.normal(size=d)
    a = rng.normal(size=(d, o)) / np.sqrt(d)
    y = np.tanh(x @ a) + 0.1 * (x[:, :o] if d >= o else 0.0) + rng.normal(size=o)
    return x, y


@pytest.mark.parametrize("n,d,o", [(256, 16, 11), (384, 7, 34)])
def test_gradients_match_the_oracle(n, d, o):
    from egspice_b200.learned import Mlp
    x, y = _data(n, d, o, 3)
    with Mlp(d, o, capacity=512, seed=11) as m:
        m.set_scaling(x, y)
        p = m.get_params()
        loss, g = m.loss_grad(x, y)
    ins, outs = om.scaling(x), om.scaling(y)
    lr, gr = om.loss_grad(p, x, y, ins, outs)
    assert abs(loss - lr) <= 1e-4 * abs(lr)
    blocks = om.unpack(np.arange(gr.size, dtype=np.float64), d, o)
    for b in blocks:
        idx = b.ravel().astype(int)
        ref, got = gr[idx], g[idx].astype(np.float64)
        err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err <= 2e-2, (b.shape, err)


def test_predictions_match_the_oracle():
    from egspice_b200.learned import Mlp
    x, y = _data(300, 16, 11, 4)
    with Mlp(16, 11, capacity=256, seed=12) as m:
        m.set_scaling(x, y)
        p = m.get_params()
        yp = m.predict(x)  # the fused kernel: three 128-row tiles, the last one partial
        yl = m.predict(x, fused=False)  # layer by layer: two chunks of the capacity
    ref = om.predict(p, x, om.scaling(x), om.scaling(y), 11)
    scale = np.abs(ref).max()
    assert np.abs(yp - ref).max() <= 2e-2 * scale
    assert np.abs(yl - ref).max() <= 2e-2 * scale
    assert np.abs(yp - yl).max() <= 1e-5 * scale


def test_training_reduces_the_loss():
    from egspice_b200.learned import Mlp, train_opts
    x, y = _data(4096, 16, 11, 5)
    with Mlp(16, 11, capacity=1024, seed=13) as m:
        losses = m.train(x, y, train_opts(epochs=40, batch=256, lr=3e-3, lr_final=3e-4))
    assert np.isfinite(losses).all()
    assert losses[-1] <= 0.1 * losses[0]


def _nominal(net):
    x0 = np.zeros((net.lanes, net.n))
    for k, v in dict(vdd=1.8, inp=0.9, vb=0.58, n1=1.2, out=0.9, tail=0.25, n2=1.2).items():
        x0[:, net.node(k)] = v
    return x0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_learned_start_points_cut_newton_iterations(oracle, precision):
    """Config-4 shape at a test size: the network is trained on the first
    2,048 points the plain method solved from the nominal start, then the
    next 1,024 points start from its predictions. With the polish on (both
    starts, and the oracle), every learned-start point meets the 1e-6 bar
    against the FP64 oracle from the nominal start and against the plain
    GPU run, in fewer Newton iterations."""
    from egspice_b200.learned import Mlp, train_opts
    polish = 6
    net = decks.miller_opamp(3072)
    opts = abi.newton_opts(init_fix=0)
    with Lanes([net], polish=polish) as L:
        L.put_x(0, _nominal(net), False)
        r0 = L.solve_static(opts)
        x_plain = L.get_x(0)
    assert ((r0[:, 0] & abi.CONVERGED) != 0).all()
    tr, te = slice(0, 2048), slice(2048, 3072)
    with Mlp(16, net.n, capacity=2048, seed=7) as m:
        m.train(net.sweep[tr], x_plain[tr], train_opts(epochs=200, batch=256, lr=3e-3, lr_final=1e-4))
        guess = m.predict(net.sweep[te])
    test = net.subset(list(range(2048, 3072)))
    with Lanes([test], precision=precision, polish=polish) as L:
        L.put_x(0, guess, False)
        r1 = L.solve_static(opts)
        x_learned = L.get_x(0)
    assert ((r1[:, 0] & abi.CONVERGED) != 0).all()
    with oracle.polish(polish):
        xo, ro = oracle.op_lanes(test, opts, x_in=_nominal(test), threads=8)
    assert (ro[:, 0] == 1).all()
    bar = lambda x, xr: float((np.abs(x - xr) / (1e-6 * np.abs(xr) + 1e-9)).max())  # noqa: E731
    assert bar(x_learned, xo) <= 1.0
    assert bar(x_learned, x_plain[te]) <= 1.0
    it_plain, it_learned = r0[te, 1].mean(), r1[:, 1].mean()
    print(f"mean Newton iterations (polished): nominal start {it_plain:.2f}, learned start {it_learned:.2f}")
    assert it_learned <= 0.8 * it_plain, (it_plain, it_learned)
