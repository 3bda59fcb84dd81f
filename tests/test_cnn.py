"""Learned initial guess: the CPU oracle of the network checked by finite
differences, the tensor-core kernels checked against the oracle (forward
values and every parameter gradient), training, and the A/B comparison with
plain extrapolation on solver-generated data.

Tolerances.  The GPU stores activations, pre-activations and gradients in
BF16 at the same points as the oracle but accumulates in float32 in another
order, and erff/expf differ from float64 in the last bits, so an occasional
BF16 rounding lands on the other side; the bars are relative L2 errors of
1e-2 for outputs and 3e-2 for each layer's weight gradient (the BF16 unit
roundoff is 3.9e-3)."""
import numpy as np
import pytest

from oracle import cnn_oracle as O

DIMS = (4, 8, 32)


def _case(seed=1, dims=DIMS):
    rng = np.random.default_rng(seed)
    theta = O.init_params(seed)
    W, b = O.unpack(theta)
    W[-1] = rng.uniform(-0.05, 0.05, size=W[-1].shape)           # a live output layer
    b = [rng.uniform(-0.1, 0.1, size=bb.shape) for bb in b]
    theta = O.pack(W, b)
    x0 = rng.standard_normal((15,) + dims)
    target = rng.standard_normal((5,) + dims)
    return theta, x0, target


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def test_oracle_gradient_matches_finite_differences():
    theta, x0, target = _case(2, (3, 4, 4))
    loss, g, _ = O.loss_and_grad(theta.astype(np.float64), x0, target, exact=True)
    rng = np.random.default_rng(0)
    th = theta.astype(np.float64)
    for idx in rng.choice(th.size, 24, replace=False):
        h = 1e-5 * max(1.0, abs(th[idx]))
        tp, tm = th.copy(), th.copy()
        tp[idx] += h
        tm[idx] -= h
        lp = O.loss_and_grad(tp, x0, target, exact=True)[0]
        lm = O.loss_and_grad(tm, x0, target, exact=True)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7, (idx, fd, g[idx])


def test_oracle_conv_transpose_is_adjoint():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((4, 3, 5, 4))
    y = rng.standard_normal((6, 3, 5, 4))
    W = rng.standard_normal((27, 6, 4))
    lhs = np.sum(O.conv(x, W) * y)
    rhs = np.sum(x * O.conv_transpose(y, W))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_parameter_layout_and_count():
    from cgli_fu_flow_b200 import cnn
    assert O.param_count() == 100357
    assert cnn.init_params(0).size == O.param_count()
    t = O.init_params(5)
    W, b = O.unpack(t)
    assert np.array_equal(O.pack(W, b), t)


# ------------------------------------------------------------------ GPU

def _net(dims=DIMS):
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.cnn import Network
    build.build()
    return Network(*dims)


@pytest.mark.gpu
def test_forward_matches_oracle():
    theta, x0, _ = _case(1)
    net = _net()
    net.set_params(theta)
    got = net.forward(x0)
    want = O.forward(theta.astype(np.float64), x0)
    err = rel_l2(got, want)
    print("forward relative L2", err)
    assert np.isfinite(got).all() and err <= 1e-2


@pytest.mark.gpu
def test_gradients_match_oracle():
    theta, x0, target = _case(4)
    net = _net()
    net.set_params(theta)
    loss, g = net.loss_grad(x0, target)
    lo, go, _ = O.loss_and_grad(theta.astype(np.float64), x0, target)
    assert abs(loss - lo) <= 1e-3 * lo
    off = 0
    for l, (ci, co) in enumerate(zip(O.CIN, O.COUT)):
        nw = 27 * ci * co
        ew = rel_l2(g[off:off + nw], go[off:off + nw])
        eb = rel_l2(g[off + nw:off + nw + co], go[off + nw:off + nw + co])
        print(f"layer {l}: dW rel L2 {ew:.2e}, db rel L2 {eb:.2e}")
        assert ew <= 3e-2 and eb <= 3e-2, l
        off += nw + co


@pytest.mark.gpu
def test_gradients_on_a_larger_grid():
    """Several CTAs per layer, more than one x chunk, wall and periodic
    halos of a longer grid."""
    dims = (40, 12, 64)
    theta, x0, target = _case(7, dims)
    net = _net(dims)
    net.set_params(theta)
    got = net.forward(x0)
    assert rel_l2(got, O.forward(theta.astype(np.float64), x0)) <= 1e-2
    loss, g = net.loss_grad(x0, target)
    lo, go, _ = O.loss_and_grad(theta.astype(np.float64), x0, target)
    assert abs(loss - lo) <= 1e-3 * lo
    assert rel_l2(g, go) <= 3e-2


@pytest.mark.gpu
def test_training_reduces_loss_on_a_fixed_pair():
    """Adam on the GPU kernels fits a smooth synthetic target."""
    dims = DIMS
    rng = np.random.default_rng(9)
    net = _net(dims)
    theta = O.init_params(0)
    net.set_params(theta)
    x0 = rng.standard_normal((15,) + dims)
    target = 0.5 * np.tanh(x0[:5] + 0.5 * x0[5:10])
    th = theta.astype(np.float32).copy()
    m = np.zeros_like(th); v = np.zeros_like(th)
    l0, _ = net.loss_grad(x0, target)
    for step in range(1, 61):
        net.set_params(th)
        loss, g = net.loss_grad(x0, target)
        O.adam(th, g, m, v, step, 3e-3)
    net.set_params(th)
    l1, _ = net.loss_grad(x0, target)
    print("loss", l0, "->", l1)
    assert l1 < 0.75 * l0


CAP = 200


@pytest.mark.gpu
def test_training_on_solver_levels_and_ab_against_extrapolation():
    """Solver A steps the seeded channel with second-order extrapolation
    while the network stores its converged levels; the network is trained
    on the GPU (Adam, own kernels) on those pairs.  Then, on held-out steps,
    a second solver B is set to A's state before every step (same levels,
    norm maxima and force) and takes the same step with the learned guess:
    an A/B test of the initial guess alone.  The learned guess must be
    closer to the converged Q^(n+1) than extrapolation and must need fewer
    inner iterations in total to reach the same stopping rule (every norm
    below 1e-3 of its running maximum; the cap of 200 is not reached on
    this 64^3 channel, unlike the reference's 30 on the smallest grids)."""
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.channel import Channel
    from cgli_fu_flow_b200.cnn import Network, init_params, physical_levels, scales_from_levels
    from cgli_fu_flow_b200.solver import Solver
    build.build()
    ch = Channel(64, 64, 64)
    A, B = Solver(ch), Solver(ch)
    A.init()
    A.set_predictor(1)
    net = Network(ch.nx, ch.ny, ch.nz)
    net.reserve_levels(64)
    net.set_params(init_params(0))
    host_levels = []
    warm, train_steps = 8, 48
    for k in range(warm + train_steps):
        A.step(None, 1e-3, CAP)
        if k >= warm:
            net.push_level(A)
            host_levels.append(physical_levels(A))
    net.set_scales(*scales_from_levels(host_levels))
    npairs = net.levels - 3
    loss0 = np.mean([net.pair_loss(p) for p in range(npairs)])
    loss = net.train(600, 1e-3, 1234, 0, npairs)
    loss1 = np.mean([net.pair_loss(p) for p in range(npairs)])
    print(f"training pairs {npairs}: loss {loss0:.4f} -> {loss1:.4f} (last mean {loss:.4f})")
    assert loss1 < 0.7 * loss0
    B.set_learned_guess(net)
    it_a, it_b, held_cnn, held_ext = [], [], [], []
    for k in range(12):
        B.copy_state_from(A)
        B.set_predictor(2)
        nb, _ = B.step(None, 1e-3, CAP)
        na, _ = A.step(None, 1e-3, CAP)
        it_a.append(na)
        it_b.append(nb)
        net.push_level(A)
        p = net.levels - 4
        held_cnn.append(net.pair_loss(p))
        q = [np.asarray(x) for x in host_levels[-3:]] + [physical_levels(A)]
        host_levels.append(q[-1])
        osc = scales_from_levels(host_levels[:train_steps])[-1]
        r = (q[3] - (3 * q[2] - 3 * q[1] + q[0])) / osc[:, None, None, None]
        held_ext.append(float(np.mean(r * r)))
    print("held-out guess MSE (normalised): learned", np.mean(held_cnn), "extrapolation", np.mean(held_ext))
    print("inner iterations from the same states: extrapolation", it_a, "learned", it_b)
    assert np.mean(held_cnn) < 0.9 * np.mean(held_ext)
    assert sum(it_b) < sum(it_a), (it_a, it_b)
    for s in (A, B):
        s.close()
    net.close()


TIGHT_DROP = 1e-8      # every norm below 1e-8 of its running maximum
STATE_TOL = 1e-6       # relative L2 per conserved variable after 100 steps


@pytest.mark.gpu
def test_mixed_learned_converges_to_the_fp64_answer_under_a_tight_rule():
    """The solution the mixed-precision + learned-guess path converges to is
    the FP64 path's: both run the same 100 physical steps from one state
    with the same stopping rule, tight enough that the stopping point no
    longer depends on the initial guess, and end within 1e-6 relative L2 of
    each other in every conserved variable.  (At the reference's loose 1e-3
    drop the two stop at different points of the inner iteration, and their
    states differ by far more: the iteration count, not the answer, is what
    the learned guess is allowed to change.)"""
    from cgli_fu_flow_b200 import build
    from cgli_fu_flow_b200.channel import Channel
    from cgli_fu_flow_b200.cnn import Network, init_params, physical_levels, scales_from_levels
    from cgli_fu_flow_b200.solver import MIXED, Solver
    build.build()
    ch = Channel(16, 16, 32)
    A = Solver(ch)
    A.init()
    A.set_predictor(1)
    net = Network(ch.nx, ch.ny, ch.nz)
    net.reserve_levels(64)
    net.set_params(init_params(0))
    host = []
    for k in range(8 + 48):
        A.step(None, 1e-3, 30)
        if k >= 8:
            net.push_level(A)
            host.append(physical_levels(A))
    net.set_scales(*scales_from_levels(host))
    net.train(600, 1e-3, 1234, 0, net.levels - 3)
    sl = np.s_[:, 3:ch.nx + 3, 2:ch.ny + 2, 2:ch.nz + 2]
    runs = {}
    for name, prec, pred in (("fp64", 0, 0), ("mixed_learned", MIXED, 2)):
        s = Solver(ch, prec)
        s.copy_state_from(A)
        if pred == 2:
            s.set_learned_guess(net)
        s.set_predictor(pred)
        its = [s.step(None, TIGHT_DROP, 400)[0] for _ in range(100)]
        runs[name] = (s.q()[sl], its)
        s.close()
    (qf, itf), (qm, itm) = runs["fp64"], runs["mixed_learned"]
    errs = [float(np.linalg.norm(qm[v] - qf[v]) / np.linalg.norm(qf[v])) for v in range(5)]
    print("mean inner iterations: fp64", np.mean(itf), "mixed + learned", np.mean(itm))
    print("state relative L2, mixed + learned vs fp64, per variable:", errs)
    assert max(itf) < 400 and max(itm) < 400, "the tight rule must be met, not capped"
    assert max(errs) <= STATE_TOL
    A.close()
    net.close()
