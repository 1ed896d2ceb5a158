"""The learned surrogate: forward and gradients of the library's kernels
against the float64 oracle (oracle/mlp_oracle.py), a training run, and the
control-variate estimator against the plain one (what the network gains)."""
import numpy as np
import pytest

from conftest import load_hbuild_case

pytestmark = pytest.mark.gpu
AUTOCM = 2.194746313e5


@pytest.fixture(scope="module")
def sur():
    import torch
    assert torch.cuda.is_available()
    from scp3_b200 import surrogate
    return surrogate


def test_forward_and_gradients_match_oracle(sur):
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(0)
    net = sur.MLP(48, hidden=256, max_batch=256, seed=3)
    net.set_output(0.02, -0.06)
    q = rng.normal(scale=np.sqrt(0.5), size=(128, 48)).astype(np.float32)
    t = (-0.06 + 0.02 * np.tanh(q[:, :4].sum(1))).astype(np.float32)
    p = net.get_params()
    y = net(q)
    y_or, _ = mo.forward(p, q, 48, 256, 0.02, -0.06)
    assert np.allclose(y, y_or, rtol=2e-3, atol=1e-5), np.abs(y - y_or).max()
    loss, g = net.loss_and_grad(q, t)
    loss_or, g_or = mo.loss_and_grad(p, q, t, 48, 256, 0.02, -0.06)
    assert loss == pytest.approx(loss_or, rel=2e-3)
    err = np.linalg.norm(g - g_or) / np.linalg.norm(g_or)
    assert err <= 1e-2, err
    # per layer too (weights and biases)
    k = 0
    for o, i in ((256, 48), (256, 256), (256, 256), (1, 256)):
        for n in (o * i, o):
            seg = slice(k, k + n)
            assert np.linalg.norm(g[seg] - g_or[seg]) <= 2e-2 * np.linalg.norm(g_or[seg]) + 1e-9
            k += n


def test_forward_many_tiles_per_block_matches_oracle(sur):
    """A batch that gives every resident block of the persistent layer kernel
    several 128-row tiles (both TMEM accumulators, each reused) and ends in a
    ragged tile."""
    from oracle import mlp_oracle as mo
    rng = np.random.default_rng(4)
    m = 3 * 148 * 128 + 77
    net = sur.MLP(48, hidden=256, max_batch=1 << 16, seed=8)
    net.set_output(0.02, -0.06)
    q = rng.normal(scale=np.sqrt(0.5), size=(m, 48)).astype(np.float32)
    y = net(q)
    y_or, _ = mo.forward(net.get_params(), q, 48, 256, 0.02, -0.06)
    assert y.shape == (m,) and np.all(np.isfinite(y))
    assert np.allclose(y, y_or, rtol=2e-3, atol=1e-5), np.abs(y - y_or).max()


def test_training_fits_a_smooth_function(sur):
    rng = np.random.default_rng(1)
    q = rng.normal(scale=np.sqrt(0.5), size=(1 << 14, 48)).astype(np.float32)
    t = (0.01 * (q[:, :8] ** 2).sum(1) - 0.002 * q[:, 0] * q[:, 1] + 0.001 * q[:, 2] ** 3).astype(np.float32)
    net = sur.MLP(48, hidden=256, max_batch=4096, seed=5)
    net.set_output(float(t.std()), float(t.mean()))
    y0 = net(q)
    before = float(np.mean((y0 - t) ** 2))
    net.fit(q, t, epochs=40, batch=1024, lr=2e-3)
    after = float(np.mean((net(q) - t) ** 2))
    assert after < 0.02 * before, (before, after)


def test_control_variate_gains_over_plain(sur):
    """Dimer doubles basis: the surrogate trained on 2^13 exact samples, then
    M_cv with 2^17 surrogate points + 2^12 exact residual points against the plain
    estimator with the same 2^12 exact points; errors of the 10 lowest levels
    compared with a 2^20-point plain build."""
    import scp3_b200
    c = load_hbuild_case("dimer_qtip4pf")

    def make(prec="bf16x3"):
        return scp3_b200.HBuild(2, c["x0"], c["MUa"], c["omega"], n2=12, n3=0, precision=prec, scramble_seed=0x5C3)

    def levels(Mraw, hb):
        M = np.asfortranarray(Mraw.copy())
        scp3_b200.ScaledMatrixElements(c["omega"], 12, 0).addHODiagonal(M)
        return np.linalg.eigvalsh(M)[:10]

    hb = make()
    qtr, vtr = sur.sample(hb, 1 << 30, 1 << 13)
    net = sur.MLP(12, hidden=256, max_batch=1 << 18, seed=9)
    net.fit(qtr, vtr.astype(np.float32), epochs=60, batch=1024, lr=2e-3)
    ref = make()
    ref.accumulate(0, 1 << 20)
    e_ref = levels(ref.read(0) / (1 << 20), ref)
    plain = make()
    plain.accumulate(0, 1 << 12)
    e_plain = levels(plain.read(0) / (1 << 12), plain)
    Mcv = sur.control_variate(make, net, 1 << 17, 1 << 12, 1 << 40, 0)
    e_cv = levels(Mcv, hb)
    err_plain = np.abs(e_plain - e_ref).max() * AUTOCM
    err_cv = np.abs(e_cv - e_ref).max() * AUTOCM
    print("levels error cm-1: plain %.3f  control variate %.3f" % (err_plain, err_cv))
    assert err_cv < err_plain


def test_builds_sharing_a_network_run_concurrently(sur):
    """Two builds with the same network attached (the two halves of the control
    variate) accumulate at the same time on their own streams: each has its own
    activation workspace, so the result equals one build after the other."""
    import scp3_b200
    c = load_hbuild_case("dimer_qtip4pf")

    def make():
        return scp3_b200.HBuild(2, c["x0"], c["MUa"], c["omega"], n2=12, n3=0, precision="bf16x3",
                                scramble_seed=0x5C3)

    net = sur.MLP(12, hidden=256, max_batch=1 << 18, seed=5)
    net.set_output(0.01, -0.01)
    seq = []
    for mode, i0 in ((sur.SURROGATE_REPLACE, 1 << 40), (sur.SURROGATE_RESIDUAL, 0)):
        hb = make()
        sur.attach(hb, net, mode)
        hb.accumulate(i0, 1 << 18)
        seq.append(hb.read(0))
        hb.close()
    a, b = make(), make()
    sur.attach(a, net, sur.SURROGATE_REPLACE)
    sur.attach(b, net, sur.SURROGATE_RESIDUAL)
    a.accumulate(1 << 40, 1 << 18)     # asynchronous: both run before either is read
    b.accumulate(0, 1 << 18)
    assert np.array_equal(a.read(0), seq[0])
    assert np.array_equal(b.read(0), seq[1])
