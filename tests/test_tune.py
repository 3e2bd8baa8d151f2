"""Autotuner host logic (CPU): candidate selection and the save / try /
restore / apply sequence, driven by a fake force path."""
import numpy as np
import pytest

from tree_b200 import api
from tree_b200.tune import Candidate, Trial, autotune, select


def test_select_fastest_within_target():
    tr = [Trial(Candidate(0.3, 0.0), 50.0, 8e-5), Trial(Candidate(0.35, 0.0), 40.0, 1.4e-4),
          Trial(Candidate(0.3, 3e-5), 42.0, 8.5e-5), Trial(Candidate(0.28, 3e-5), 42.0, 7e-5)]
    best = select(tr, 1e-4, margin=0.9)
    assert best.cand == Candidate(0.28, 3e-5)  # tie on time: lower rms wins
    assert select(tr, 1e-5) is None
    assert select([Trial(Candidate(0.3, 0.0), 1.0, float("nan"))], 1.0) is None


class FakeForce:
    """Forces = exact * (1 + c theta^4 - d eta), time = a/theta^3 - b eta."""

    def __init__(self, n=64):
        rng = np.random.default_rng(1)
        self.n_el = self.n_ion = n // 2
        self.exact = rng.standard_normal((n, 3))
        self.state = {k: rng.standard_normal((n // 2, 3)) for k in
                      ("x_el", "v_el", "f_el", "x_ion", "v_ion", "f_ion")}
        self.cfg, self.tune, self.eta, self.model = None, None, 0.0, None
        self.loads, self.t = [], api.Timing()
        self.f = self.exact.copy()

    def get_state(self):
        return {k: v.copy() for k, v in self.state.items()}

    def load_state(self, *a):
        self.loads.append(a)

    def set_config(self, cfg):
        self.cfg = cfg

    def set_tuning(self, bucket, bps, order):
        self.tune = (bucket, bps, order)

    def mac_set_model(self, p, s):
        self.model = (p, s)

    def mac_config(self, eta, lo, hi):
        self.eta = eta

    def step(self, dt, n):
        th = self.cfg.theta
        eta = self.eta if self.cfg.mac == api.MAC_LEARNED else 0.0
        self.f = self.exact * (1 + 2e-2 * th ** 4 + eta)
        self.t.ms_walk += 1.0 / th ** 3 - 1e4 * eta
        self.t.ms_build += 1.0

    def timings(self):
        t = api.Timing()
        t.ms_walk, t.ms_build = self.t.ms_walk, self.t.ms_build
        return t

    def direct(self, idx):
        return self.exact[idx], None


@pytest.fixture
def fake(monkeypatch):
    ff = FakeForce()
    orig = ff.get_state

    def gs():
        s = orig()
        s["f_el"], s["f_ion"] = ff.f[: ff.n_el].copy(), ff.f[ff.n_el:].copy()
        return s
    ff.get_state = gs
    return ff


def test_autotune_picks_fastest_accurate_and_restores(fake):
    space = [Candidate(t, e) for t in (0.2, 0.3, 0.4) for e in (0.0, 1e-5)]
    best, trials = autotune(fake, 0.1, space=space, target=2e-4, margin=1.0,
                            audit=32, model=(np.zeros(1), np.zeros(1)))
    assert len(trials) == 6
    # rms = 2e-2 theta^4 + eta: theta 0.3 -> 1.6e-4 (+1e-5 -> 1.7e-4), 0.4 -> 5.1e-4
    assert best.cand == Candidate(0.3, 1e-5)
    assert fake.cfg.theta == 0.3 and fake.cfg.mac == api.MAC_LEARNED and fake.eta == 1e-5
    assert fake.tune == (8, 4, 3)
    assert len(fake.loads) == 2 * len(space) + 1  # two loads per trial + restore


def test_autotune_skips_learned_without_model(fake):
    space = [Candidate(0.3, 0.0), Candidate(0.3, 1e-5)]
    best, trials = autotune(fake, 0.1, space=space, target=2e-4, margin=1.0, audit=16)
    assert [t.cand for t in trials] == [Candidate(0.3, 0.0)]
    assert best.cand == Candidate(0.3, 0.0)
