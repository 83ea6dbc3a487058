"""Host-side logic of the learned first-attempt delta (no GPU): how the
network's predictions become per-front deltas, and the fitted margin."""
import numpy as np

from ma57_b200 import learned


class _Fixed(learned.DeltaModel):
    """DeltaModel with a stand-in for the device network."""

    def __init__(self, pred, margin):
        self._pred = np.asarray(pred, dtype=np.float64)
        self.mean = np.zeros(learned.NFEAT)
        self.std = np.ones(learned.NFEAT)
        self.margin = margin

    def predict_log10(self, X):
        return self._pred[: len(X)]


def test_front_deltas_floor_at_median_and_plain_first_attempt():
    X = np.zeros((5, learned.NFEAT))
    m = _Fixed([-2.0, 0.5, 1.0, 3.0, 1.5], margin=0.25)
    d = m.front_deltas(X, base=1e-14)
    # each front: max(prediction, median 1.0) + margin decades above base
    expect = 1e-14 * 10.0 ** (np.maximum([-2.0, 0.5, 1.0, 3.0, 1.5], 1.0) + 0.25)
    np.testing.assert_allclose(d, expect, rtol=1e-12)


def test_front_deltas_never_below_base():
    X = np.zeros((3, learned.NFEAT))
    m = _Fixed([-4.0, -3.0, -5.0], margin=0.5)
    d = m.front_deltas(X, base=2e-12)
    np.testing.assert_array_equal(d, np.full(3, 2e-12))


def test_update_after_a_passing_first_attempt_only_buffers():
    m = _Fixed([0.0], margin=0.1)
    X = np.ones((4, learned.NFEAT))
    T = np.zeros(4)
    for _ in range(25):
        assert m.update(X, T, retries=0, window=20) is None  # nothing new to learn
    assert len(m._buf) == 20  # the window keeps the last 20 matrices
    assert m.margin == 0.1
