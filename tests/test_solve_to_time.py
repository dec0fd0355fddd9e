"""learned.solve_to_time's host logic on a stand-in context (no GPU): it ends
exactly on t_end with one step of the remaining time, never lets a batch of
CFL steps pass t_end while dt grows no faster than the assumed rate, and
reads dt back once per batch far from t_end."""
import numpy as np
import pytest

pytest.importorskip("torch")
from deepgreen import learned  # noqa: E402


class FakeContext:
    """dt of step i is dt0 * rate**i; records the calls the solve makes."""

    def __init__(self, dt0, rate):
        self.dt0, self.rate = dt0, rate
        self.steps = 0
        self.t = 0.0
        self.history = []
        self.reads = 0
        self.last_dt = None

    def _dt(self, i):
        return self.dt0 * self.rate ** i

    def next_dt(self):
        self.reads += 1
        return self._dt(self.steps)

    def enqueue_steps(self, m):
        for _ in range(m):
            d = self._dt(self.steps)
            self.history.append(d)
            self.t += d
            self.steps += 1

    def get_dts(self, m):
        self.reads += 1
        return np.array(self.history[-m:])

    def compute_step_dt(self, dt):
        self.last_dt = dt
        self.history.append(dt)
        self.t += dt
        self.steps += 1

    def synchronize(self):
        pass


@pytest.mark.parametrize("rate", [1.0, 1.05, 0.97])
def test_ends_exactly_on_t_end(rate, monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    ctx = FakeContext(1e-3, rate)
    t_end = 0.02              # reachable for every rate (0.97: the dts sum to 0.033)
    steps, _ = learned.solve_to_time(ctx, t_end)
    assert steps == ctx.steps
    assert ctx.t == pytest.approx(t_end, rel=1e-12)
    # every CFL step stayed short of the end: the sum before the last step < t_end
    assert sum(ctx.history[:-1]) < t_end
    assert ctx.last_dt is not None and 0 < ctx.last_dt <= ctx._dt(ctx.steps - 1) + 1e-15


def test_batches_far_from_the_end(monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    ctx = FakeContext(1e-3, 1.0)
    learned.solve_to_time(ctx, 1.0, batch=16)
    # ~1000 steps: one dt read and one history read per batch of 16, single
    # steps only near the end
    assert ctx.steps == 1000
    assert ctx.reads < 1000 // 16 * 2 + 40
