"""Host logic of the time-stepped inversion driver on a stand-in objective
(no GPU): a quadratic with a known minimiser stands in for
``TimeSteppedObjective`` (same call and record interface)."""
import numpy as np

from glide_b200.inverse import finite_difference_check, invert_time_stepped


class Quadratic:
    """f(x) = 1/2 (x - x*)^T D (x - x*) with the TimeSteppedObjective interface."""

    def __init__(self, n=50, seed=0, sleep=0.0):
        rng = np.random.default_rng(seed)
        self.d = rng.uniform(0.5, 20.0, n)
        self.xs = rng.uniform(-2.0, 2.0, n)
        self.evaluations = 0
        self.last = {}
        self.sleep = sleep

    def __call__(self, x):
        import time
        if self.sleep:
            time.sleep(self.sleep)
        r = np.asarray(x) - self.xs
        f = 0.5 * float(np.sum(self.d * r * r))
        self.evaluations += 1
        self.last = {"misfit": f, "reg": 0.0, "total": f}
        return f, self.d * r

    def value(self, x):
        return self(x)[0]


def test_lbfgs_reaches_the_minimiser_and_records_every_iteration():
    q = Quadratic()
    x0 = np.zeros(50)
    x, rec = invert_time_stepped(q, x0, maxiter=200, bounds=(-6.0, 5.0))
    assert np.max(np.abs(x - q.xs)) <= 1e-4
    assert rec["iterations"] == len(rec["misfit_total_per_iteration"]) >= 2
    assert not rec["stopped_on_time"]
    assert rec["final_total"] <= 1e-8 * rec["initial"]["total"]
    totals = [t for _, t in rec["misfit_total_per_iteration"]]
    assert all(b <= a * (1 + 1e-12) for a, b in zip(totals, totals[1:]))


def test_lbfgs_wall_time_cap_returns_the_last_accepted_iterate():
    q = Quadratic(sleep=0.02)
    x, rec = invert_time_stepped(q, np.zeros(50), maxiter=200, max_seconds=0.1)
    assert rec["stopped_on_time"]
    assert 1 <= rec["iterations"] < 200
    # the returned point is the last accepted iterate, with the recorded objective
    assert abs(q(x)[0] - rec["final_total"]) <= 1e-12 * max(1.0, rec["final_total"])


def test_finite_difference_check_on_a_smooth_objective():
    q = Quadratic(n=20, seed=3)
    x = np.zeros(20)
    _, g = q(x)
    errs, pairs, smooth = finite_difference_check(q, x, n_directions=4, eps=1e-6, grads=[g, 2.0 * g],
                                                  smooth_dirs=2)
    assert max(errs[0]) <= 1e-6          # the true gradient
    assert min(errs[1]) >= 0.99          # twice the gradient: off by 100 %
    assert len(smooth) == 2 and max(smooth) <= 1e-6
    assert all(len(p) == 3 for p in pairs)
