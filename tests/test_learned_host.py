"""Host-side logic of the learned sketch-rank method (no GPU): the feature
vector of a (kind, bond) and the proposal rule ell = max(ceil(pred),
r_prev + 1) + pad clamped to [pad + 1, maxrank + pad]."""
import numpy as np

from paratt_b200 import KINDS, STAT_NSIG
from paratt_b200 import learned as L


def test_features_layout():
    d, dt, delta = 5, 1e-3, 1e-6
    sig = np.zeros((d + 1, STAT_NSIG))
    sig[2, :3] = [1e-6, 1e-2, 1e30]  # at delta, 4 decades above, clipped high
    f = L.features(sig, delta, d, dt, kind=1)
    assert f.shape == (d - 1, L.NIN) and f.dtype == np.float32
    row = f[1]  # bond 2
    np.testing.assert_allclose(row[:3], [0.0, 1.0, 4.0], atol=1e-7)
    assert row[3] == -1.0  # zero singular values clip at -4, scaled by 1/4
    np.testing.assert_allclose(f[:, STAT_NSIG], np.arange(1, d) / d, rtol=1e-6)
    np.testing.assert_allclose(f[:, STAT_NSIG + 1], np.log10(dt) + 3.0, atol=1e-7)
    onehot = f[:, STAT_NSIG + 2:]
    assert onehot.shape[1] == KINDS
    assert (onehot[:, 1] == 1.0).all() and (onehot.sum(axis=1) == 1.0).all()


class _FixedMLP:
    def __init__(self, values):
        self.values = np.asarray(values, dtype=np.float32)

    def forward(self, x):
        assert x.shape[1] == L.NIN
        return np.resize(self.values, x.shape[0])


def test_proposal_rail_and_clamp():
    d, pad, maxrank = 4, 4, 10
    specs = [(np.ones((d + 1, STAT_NSIG)), 1e-8)] * KINDS
    mlp = _FixedMLP([2.2, 0.1, 30.0])  # per bond, repeated over the kinds
    prev = np.array([[1, 5, 1, 3, 1]] * KINDS)
    ell = L.propose(mlp, specs, d, 1e-3, pad, maxrank, prev=prev)
    assert ell.shape == (KINDS, d + 1)
    assert (ell[:, 0] == 1).all() and (ell[:, -1] == 1).all()
    # bond 1: ceil(2.2) = 3 < prev 5 + 1 -> 6, + pad
    # bond 2: ceil(0.1) = 1, prev 1 + 1 = 2 -> 2, + pad
    # bond 3: ceil(30) = 30 -> clamped to maxrank + pad
    assert ell[0, 1:d].tolist() == [6 + pad, 2 + pad, maxrank + pad]
    # without the rail only the clamp applies
    ell2 = L.propose(mlp, specs, d, 1e-3, pad, maxrank)
    assert ell2[0, 1:d].tolist() == [3 + pad, 1 + pad, maxrank + pad]
