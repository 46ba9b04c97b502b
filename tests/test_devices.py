"""Device models of the oracle against central finite differences (the
reference's jacobian_fd tests, src/device/tests/jacobian_fd.zig, need VerA;
the restated models are pinned here the same way), the limiters against
their published ngspice semantics, and the MC sampler's golden hooks."""
import numpy as np
import pytest

from egspice_b200 import decks


def fd_check(oracle, net, b, inst, v, rtol=2e-5, atol=1e-13):
    f0, j0, q0, c0 = oracle.device_probe(net, b, inst, 0, v)
    nt = len(v)
    for c in range(nt):
        h = 1e-7 * max(1.0, abs(v[c]))
        vp = np.array(v, float)
        vm = np.array(v, float)
        vp[c] += h
        vm[c] -= h
        fp = oracle.device_probe(net, b, inst, 0, vp)
        fm = oracle.device_probe(net, b, inst, 0, vm)
        dfd = (fp[0] - fm[0]) / (2 * h)
        dq = (fp[2] - fm[2]) / (2 * h)
        for r in range(nt):
            assert abs(dfd[r] - j0[r, c]) <= rtol * max(abs(dfd[r]), abs(j0[r, c])) + atol, (r, c, dfd[r], j0[r, c])
            assert abs(dq[r] - c0[r, c]) <= rtol * max(abs(dq[r]), abs(c0[r, c])) + 1e-22, (r, c)


@pytest.mark.parametrize("bias", [
    (1.0, 1.2, 0.0, 0.0),    # NMOS saturation
    (0.2, 1.5, 0.0, 0.0),    # linear
    (0.5, 0.3, 0.0, 0.0),    # cutoff
    (-0.4, 1.0, 0.0, -0.3),  # reverse mode, body biased
    (0.7, 1.1, 0.2, 0.35),   # forward-biased bulk (sbody continuation)
])
def test_mos1_jacobian_fd(oracle, bias):
    # Above vbx = 0 the body root is Taylor-continued and its slope is
    # ngspice's gm*gamma/(2 sarg), not the continuation's own slope
    # (models/mos1.va:323-334): there the finite difference of the value is
    # not the model's Jacobian, so those biases run without body effect.
    vd, vg, vs, vb = bias
    vds = vd - vs
    vbx = (vb - vs) if vds >= 0 else (vb - vd)
    gam = 0.4 if vbx <= 0 else 0.0
    b = decks.Builder("m", 1)
    b.m("d", "g", "s", "b", 1.0, 0.45, 200e-6, 2e-6, 0.18e-6, gamma=gam, phi=0.7, lam=0.05)
    net = b.freeze()
    fd_check(oracle, net, 0, 0, list(bias))
    b = decks.Builder("p", 1)
    b.m("d", "g", "s", "b", -1.0, -0.45, 80e-6, 4e-6, 0.18e-6, gamma=gam, phi=0.7, lam=0.04)
    net = b.freeze()
    fd_check(oracle, net, 0, 0, [-x for x in bias])


@pytest.mark.parametrize("vd", [-0.5, -0.01, 0.0, 0.3, 0.65, 0.8])
def test_diode_jacobian_fd(oracle, vd):
    b = decks.Builder("d", 1)
    b.d("a", "0", cjo=1e-12, tt=1e-10)
    net = b.freeze()
    fd_check(oracle, net, 0, 0, [vd, 0.0], rtol=1e-4, atol=1e-15)


def test_pnjlim(oracle):
    import ctypes
    L = oracle.lib()
    chk = ctypes.c_int(0)
    vt, vcrit = 0.025851991, 0.6
    assert L.orc_pnjlim(0.5, 0.4, vt, vcrit, ctypes.byref(chk)) == 0.5 and chk.value == 0
    v = L.orc_pnjlim(1.5, 0.6, vt, vcrit, ctypes.byref(chk))
    assert chk.value == 1 and abs(v - (0.6 + vt * np.log(1 + 0.9 / vt))) < 1e-15
    v = L.orc_pnjlim(1.5, -0.2, vt, vcrit, ctypes.byref(chk))
    assert chk.value == 1 and abs(v - vt * np.log(1.5 / vt)) < 1e-15
    v = L.orc_pnjlim(-5.0, 0.3, vt, vcrit, ctypes.byref(chk))
    assert v == -1.3 and chk.value == 1


def test_fetlim_limvds(oracle):
    L = oracle.lib()
    assert L.orc_limvds(10.0, 1.0) == 4.0
    assert L.orc_limvds(-3.0, 1.0) == -0.5
    assert L.orc_limvds(20.0, 4.0) == 14.0
    assert L.orc_limvds(1.0, 4.0) == 2.0
    vto = 0.45
    assert L.orc_fetlim(5.0, 0.0, vto) == vto + 0.5      # off, turning on: clamp
    assert L.orc_fetlim(0.3, 0.0, vto) == 0.3
    assert L.orc_fetlim(10.0, 1.0, vto) == vto + 4       # middle region rising
    assert L.orc_fetlim(-10.0, 5.0, vto) == vto + 2      # on, going off past vtox


def test_sampler_golden_hooks(oracle):
    """siteKey and normalQuantile: the Python sampler equals the C
    restatement bit for bit, and the quantile round-trips the normal CDF."""
    L = oracle.lib()
    rng = np.random.default_rng(5)
    for _ in range(200):
        a, b = (int(v) for v in rng.integers(0, 2**63, 2, dtype=np.int64))
        assert int(decks.site_key(np.uint64(a), np.uint64(b))) == L.orc_site_key(a, b)
    from math import erf, sqrt
    for u in np.concatenate([np.linspace(1e-6, 1 - 1e-6, 101), [0.01, 0.02425, 0.5, 0.97575]]):
        x = float(decks.normal_quantile(np.array([u]))[0])
        assert x == L.orc_normal_quantile(float(u))
        assert abs(0.5 * (1 + erf(x / sqrt(2))) - u) < 2e-9


def test_points_depend_only_on_their_index():
    a = decks.inverter_chain(8, first_point=0)
    b = decks.inverter_chain(4, first_point=4)
    for ba, bb in zip(a.batches, b.batches):
        assert np.array_equal(ba.param[:, :, 4:], bb.param)


def test_pulse_waveform():
    from egspice_b200.decks import _src_params
    p = _src_params(0.0, (0.0, 1.0, 1e-9, 1e-9, 2e-9, 3e-9, 10e-9))
    assert p[1] == 1.0
