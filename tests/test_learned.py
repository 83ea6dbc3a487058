"""The learned first-attempt delta: the CUDA network's gradient against the
CPU oracle (oracle/mlp_ref.py), GPU training against the oracle's Adam, and
what the trained network gains over plain escalation on an interior-point
sequence (config 5's construction on a smaller grid)."""
import math

import numpy as np
import pytest

from ma57_b200 import Mode, OrderingType, RefinementOptions, SymLDLT
from ma57_b200 import learned
from ma57_b200 import matrices as M
from oracle import mlp_ref as R

pytestmark = pytest.mark.gpu


def test_gradient_matches_cpu_oracle():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((3000, R.IN))
    T = rng.standard_normal(3000)
    p = learned.init_params(4) + 0.1 * rng.standard_normal(R.P)
    net = learned.Network(p)
    loss, g = net.gradient(X, T)
    loss_ref, g_ref = R.loss_and_grad(p, X, T)
    assert abs(loss - loss_ref) <= 1e-12 * loss_ref
    assert np.abs(g - g_ref).max() <= 1e-12 * max(1.0, np.abs(g_ref).max())
    y = net.predict(X)
    np.testing.assert_allclose(y, R.forward(p, X)[0], rtol=0, atol=1e-12)


def test_gpu_training_matches_cpu_adam():
    rng = np.random.default_rng(2)
    X = rng.standard_normal((2048, R.IN))
    T = np.tanh(X[:, 0] - 0.5 * X[:, 3]) + 0.1 * X[:, 5]
    p0 = learned.init_params(8)
    net = learned.Network(p0)
    loss = net.train(X, T, epochs=30, lr=1e-2, minibatch=512)
    p_ref = R.adam(p0, X, T, epochs=30, lr=1e-2, minibatch=512)
    assert np.abs(net.params() - p_ref).max() <= 1e-9
    assert loss < 0.5 * R.loss_and_grad(p0, X, T)[0]


def _run(seq, steps, model=None, initial=1e-14):
    """Factorize each step in StaticRegularized mode from a small first delta
    (plain escalation x10 on a failed inertia check), refine towards 1e-10.
    Returns retries and refined residuals per step, feature rows and the
    accepted deltas in decades above the first attempt (training targets)."""
    s = SymLDLT()
    s.setMode(Mode.StaticRegularized)
    s.setOrdering(OrderingType.AMD)
    s.setKKTBlockSizes(seq.n1, seq.n2)
    s.setMaxRegularizationRetries(40)
    retries, resid, feats, targets = [], [], [], []
    signs = np.r_[-np.ones(seq.n1), np.ones(seq.n2)]
    sym = None
    for step in steps:
        K, _ = seq.matrix(step)
        if sym is None:
            s.analyzePattern(K)
            sym = s.symbolicFactor()
        base = initial * abs(K.data).max()
        s.setInitialRegularizationDelta(base)
        F = learned.front_features(sym, K, signs)
        s.setFrontDeltas(None if model is None else model.front_deltas(F, base))
        s.factorize(K)
        r = s.solveWithRefinement(K, seq.b, RefinementOptions(max_iterations=30, tolerance=1e-10))
        retries.append(s.regularizationRetriesUsed())
        resid.append(r.diagnostics.final_relative_residual)
        feats.append(F)
        targets.append(np.full(F.shape[0], math.log10(s.lastRegularizationDelta() / base)))
    return retries, resid, feats, targets


def test_config5_as_specified_needs_no_retries():
    """K_k = [[-E_k, A^T], [A, F_k]] with E_k positive definite and F_k > 0 is
    symmetric quasi-definite: every pivot has its expected sign, so plain
    escalation never retries (there is nothing for a learned delta to cut)."""
    seq = M.InteriorPointSequence(k=10, steps=60)
    retries, resid, _, _ = _run(seq, range(0, 60, 6))
    assert max(retries) == 0
    assert max(resid) <= 1e-10


def test_learned_delta_cuts_retries_on_nonconvex_sequence():
    """With negative curvature (E_k = L7 - 6 I + diag(mu_k / x^2)) the
    inertia check fails until delta is large enough; the network, trained on
    the deltas escalation accepted for the first 30 matrices, predicts the
    first attempt for the next 30."""
    seq = M.InteriorPointSequence(k=10, steps=60, curvature_shift=6.0)
    _, _, feats, targets = _run(seq, range(0, 30))
    model = learned.DeltaModel(seed=3)
    groups = np.concatenate([np.full(len(t), i) for i, t in enumerate(targets)])
    model.fit(np.vstack(feats), np.concatenate(targets), groups, epochs=300, lr=3e-3, minibatch=2048)
    state = (seq.logx.copy(), seq.st.pos)
    plain, plain_res, _, _ = _run(seq, range(30, 60))
    seq.logx, seq.st.pos = state
    with_model, model_res, _, _ = _run(seq, range(30, 60), model=model)
    assert np.mean(plain) >= 5
    assert np.mean(with_model) <= 0.5 * np.mean(plain)
    for a, b in zip(model_res, plain_res):
        assert a <= max(10 * b, 1e-10)


def test_failed_learned_attempt_resumes_escalation_above_it():
    """A per-front first attempt that fails the inertia check costs one
    attempt: the escalation resumes one growth step above the smallest
    delta it used, not from the initial delta."""
    seq = M.InteriorPointSequence(k=10, steps=60, curvature_shift=6.0)
    K, _ = seq.matrix(0)
    base = 1e-14 * abs(K.data).max()

    def run(front):
        s = SymLDLT()
        s.setMode(Mode.StaticRegularized)
        s.setOrdering(OrderingType.AMD)
        s.setKKTBlockSizes(seq.n1, seq.n2)
        s.setMaxRegularizationRetries(40)
        s.analyzePattern(K)
        s.setInitialRegularizationDelta(base)
        if front is not None:
            s.setFrontDeltas(np.full(len(s.symbolicFactor().supernodes), front))
        s.factorize(K)
        return s.regularizationRetriesUsed(), s.lastRegularizationDelta(), s.inertia().as_tuple()

    plain_retries, plain_delta, inertia = run(None)
    assert plain_retries >= 2
    # a first attempt j decades above the initial delta, still too small
    j = max(1, plain_retries - 2)
    retries, delta, inertia2 = run(base * 10.0**j)
    assert inertia2 == inertia == (seq.n2, seq.n1, 0)
    assert retries == plain_retries - j
    assert delta == pytest.approx(plain_delta, rel=1e-9)
