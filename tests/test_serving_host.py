"""The stream driver against a host-side model of the server (no GPU): FIFO
admission into a bounded number of slots, iterations advanced per step,
latency counted from arrival to the step that finished the request."""
import numpy as np

from softdft_b200.serving import poisson_arrivals, serve_stream


class FakeServer:
    def __init__(self, slots, need):
        self.slots, self.need = slots, need
        self.queue, self.active, self.done = [], {}, []
        self.admit_order = []

    def submit(self, system, tag):
        self.queue.append(tag)

    def step(self, iters):
        while self.queue and len(self.active) < self.slots:
            t = self.queue.pop(0)
            self.admit_order.append(t)
            self.active[t] = 0
        for t in list(self.active):
            self.active[t] += iters
            if self.active[t] >= self.need[t]:
                self.done.append((t, 0, self.need[t], 1e-9, 0.0))
                del self.active[t]
        return len(self.active), len(self.queue)

    def poll(self):
        out, self.done = self.done, []
        return out


class Clock:
    """Simulated time: every step costs 1 ms, sleeping advances the clock."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, d):
        self.t += d


def test_poisson_arrivals_are_seeded_and_increasing():
    a = poisson_arrivals(1000, 200.0, seed=3)
    assert np.all(np.diff(a) > 0)
    assert np.array_equal(a, poisson_arrivals(1000, 200.0, seed=3))
    assert abs(1000 / a[-1] - 200.0) < 30.0


def test_stream_completes_in_fifo_order_with_bounded_slots():
    n = 40
    need = {i: 5 + (i % 7) * 3 for i in range(n)}
    srv = FakeServer(slots=4, need=need)
    clock = Clock()

    class Stepper:
        def submit(self, s, t):
            srv.submit(s, t)

        def step(self, it):
            clock.t += 1e-3
            return srv.step(it)

        def poll(self):
            return srv.poll()

    arrivals = np.linspace(0.0, 0.01, n)
    res = serve_stream(Stepper(), [None] * n, arrivals, iters_per_step=5, clock=clock, sleep=clock.sleep)
    assert res["n"] == n and np.all(res["status"] == 0)
    assert srv.admit_order == list(range(n))
    assert np.all(res["iters"] == np.array([need[i] for i in range(n)]))
    assert np.all(res["latency_ms"] > 0)
    assert res["p99_ms"] >= res["p50_ms"]


def test_idle_server_waits_for_the_next_arrival():
    srv = FakeServer(slots=2, need={0: 1, 1: 1})
    clock = Clock()

    class Stepper:
        def submit(self, s, t):
            srv.submit(s, t)

        def step(self, it):
            clock.t += 1e-3
            return srv.step(it)

        def poll(self):
            return srv.poll()

    res = serve_stream(Stepper(), [None, None], [0.0, 5.0], iters_per_step=1, clock=clock, sleep=clock.sleep)
    # the second request waits for its own arrival, not for the first one
    assert res["latency_ms"][1] < 10.0 and res["wall_s"] >= 5.0
