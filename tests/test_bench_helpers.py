"""Host-side helpers of bench.py (no GPU): the equal-accuracy fit of the plain
FP64 arms and the workload description both arms print."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_equal_accuracy_recovers_power_laws():
    # rms = 0.04 theta^3, ms = 50 theta^-3: rms 1e-4 at theta = (1/400)^(1/3)
    pts = [(th, 0.04 * th ** 3, 50.0 * th ** -3) for th in (0.5, 0.35, 0.25)]
    eq = bench.equal_accuracy(pts, 1e-4)
    want = (1e-4 / 0.04) ** (1 / 3)
    assert eq["theta"] == pytest.approx(want, rel=1e-9)
    assert eq["ms_per_step"] == pytest.approx(50.0 * want ** -3, rel=1e-9)
    assert eq["rms_exponent"] == pytest.approx(3.0) and eq["extrapolated"]


def test_equal_accuracy_needs_two_usable_points():
    assert bench.equal_accuracy([(0.5, 1e-2, 100.0)]) is None
    assert bench.equal_accuracy([(0.5, None, 100.0), (0.3, 1e-3, 300.0)]) is None
    # error growing as theta shrinks: no crossing to report
    assert bench.equal_accuracy([(0.5, 1e-3, 100.0), (0.3, 1e-2, 300.0)]) is None


def test_equal_accuracy_refuses_nonmonotone_or_far_fits():
    # the error rises between two of the arms: no trend to follow
    pts = [(0.5, 1.0e-2, 295.0), (0.35, 1.6e-2, 606.0), (0.25, 5.1e-3, 1293.0)]
    assert bench.equal_accuracy(pts, 1e-4) is None
    # a steady trend whose crossing lies far below the smallest arm
    pts = [(0.5, 1.0e-2, 100.0), (0.25, 9.0e-3, 400.0)]
    assert bench.equal_accuracy(pts, 1e-4) is None


def test_both_arms_describe_the_same_workload():
    import argparse
    args = argparse.Namespace(te=50.0, theta=0.3, physics="kelbg", no_rdf=False, nsamp=10)
    a = bench.workload_config(args, 1048576)
    b = bench.workload_config(args, 1048576)
    assert a == b and a["rdf"] and a["n_particles"] == 1048576
    assert not {"precision", "mac", "eta", "order", "bucket"} & set(a)


def test_whole_job_rate():
    assert bench.whole_job_rate(1000, 2, 10, 20.0) == pytest.approx(1e6)
    assert np.isfinite(bench.whole_job_rate(1, 1, 1, 1e-3))


class _FakeEnsemble:
    """Two clouds whose forces differ from their direct sums by known
    relative errors: cloud 0 by 1e-4 on every particle, cloud 1 by 3e-4."""

    def __init__(self):
        self.offsets = np.array([0, 5000, 11000])
        rng = np.random.default_rng(3)
        self.fd = rng.standard_normal((11000, 3)) + 2.0
        scale = np.where(np.arange(11000) < 5000, 1e-4, 3e-4)[:, None]
        unit = rng.standard_normal((11000, 3))
        unit /= np.linalg.norm(unit, axis=1)[:, None]
        self.f = self.fd + scale * np.linalg.norm(self.fd, axis=1)[:, None] * unit

    def get_state(self):
        return {"f": self.f}

    def direct(self, cloud, targets):
        a = int(self.offsets[cloud])
        return self.fd[a + np.asarray(targets)], None


def test_ensemble_rms_is_per_cloud():
    rms = bench.ensemble_rms(_FakeEnsemble(), 2)
    assert rms == pytest.approx([1e-4, 3e-4], rel=1e-9)
