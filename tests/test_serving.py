"""The continuous-batching serving loop (iccg_b200.batch.ServingLoop) on the
CPU, with stand-ins for the batch, the contexts and the device memory:
admission by free memory and budget, requests admitted while others run,
retirement between steps, failures reported with their cause."""
from types import SimpleNamespace

import numpy as np

import iccg_b200.batch as bt


class _Ctx:
    made = 0

    def __init__(self, device):
        _Ctx.made += 1
        self.n = 0
        self.device_bytes = 0
        self.closed = False

    def close(self):
        self.closed = True


def _load(ctx, P, storage):
    if getattr(P, "bad", False):
        raise RuntimeError("IC(0) pivot <= 0 at row 3")
    ctx.n = P.n
    ctx.device_bytes = 100 * P.n
    ctx.P = P


class _Batch:
    """Solve s stops after P.steps steps; results carry the slot's system."""

    def __init__(self, device):
        self.systems = {}
        self.slots = {}
        self.next_sys = 0
        self.max_running = 0
        self.open_args = None
        self.steps = 0

    def open(self, slots, storage, rr_interval=50, graph_iters=8):
        self.open_args = (slots, storage, graph_iters)
        self.cap = slots

    def add_system(self, ctx):
        k = self.next_sys
        self.next_sys += 1
        self.systems[k] = ctx
        return k

    def remove_system(self, k):
        assert all(v["sys"] != k for v in self.slots.values())
        del self.systems[k]

    def submit(self, k, b, x0, max_iter, tol):
        assert len(self.slots) < self.cap
        s = min(set(range(self.cap)) - set(self.slots))
        self.slots[s] = {"sys": k, "left": self.systems[k].P.steps, "stopped": False}
        return s

    def step(self):
        import time
        time.sleep(0.001)                             # the device's time for the step
        self.steps += 1
        running = [v for v in self.slots.values() if not v["stopped"]]
        self.max_running = max(self.max_running, len(running))
        out = []
        for s, v in self.slots.items():
            if v["stopped"]:
                continue
            v["left"] -= 1
            if v["left"] <= 0:
                v["stopped"] = True
                out.append(s)
        return out, len(running) - len(out)

    def retire(self, slots):
        res = []
        for s in slots:
            v = self.slots.pop(s)
            P = self.systems[v["sys"]].P
            ok = not getattr(P, "diverge", False)
            res.append(SimpleNamespace(converged=ok, iters=4 * P.steps, status="converged" if ok else "max_iter",
                                       solve_ms=0.5))
        return [np.zeros(1)] * len(slots), res

    def close(self):
        pass


def _req(i, t, n=100, steps=3, est=1000, **kw):
    return bt.Request(i, t, (lambda: SimpleNamespace(n=n, steps=steps, b_run=np.zeros(n), **kw)), est)


def _loop(batch, **kw):
    args = dict(budget_bytes=10**6, slots=64, builders=2, reserve_bytes=0, graph_iters=4,
                make_batch=lambda dev: batch, make_context=_Ctx, load=_load, free_memory=lambda dev: 10**9)
    args.update(kw)
    return bt.ServingLoop(**args)


def test_every_request_served_and_overlapping():
    B = _Batch(0)
    reqs = [_req(i, 0.001 * i, steps=5 + i % 3) for i in range(20)]
    st = _loop(B).run(reqs)
    s = st.summary()
    assert s["solves"] == 20 and s["failed"] == 0
    assert s["p99_ms"] >= s["p50_ms"] > 0 and s["solves_per_s"] > 0
    # continuous batching: later requests joined while earlier ones ran
    assert B.max_running > 1 and st.max_in_flight > 1
    assert B.open_args == (64, bt.STORE_FP32, 4)
    assert not B.slots and not B.systems          # all retired, systems taken out


def test_failures_are_reported_with_their_cause():
    B = _Batch(0)
    reqs = [_req(0, 0.0), _req(1, 0.0, bad=True), _req(2, 0.0, diverge=True), _req(3, 0.001)]
    st = _loop(B).run(reqs)
    assert st.failed == 2 and len(st.latencies_ms) == 2
    assert any("request 1" in e and "pivot" in e for e in st.errors)
    assert any("request 2" in e and "max_iter" in e for e in st.errors)
    assert "errors" in st.summary()


def test_budget_limits_what_is_in_flight():
    B = _Batch(0)
    reqs = [_req(i, 0.0, steps=4, est=400) for i in range(10)]
    st = _loop(B, budget_bytes=1000).run(reqs)           # two at a time fit
    assert st.summary()["solves"] == 10
    assert B.max_running <= 2


def test_free_device_memory_limits_admission():
    B = _Batch(0)
    live = []

    def make_ctx(dev):
        c = _Ctx(dev)
        live.append(c)
        return c

    def load(ctx, P, storage):
        _load(ctx, P, storage)
        ctx.device_bytes = 400

    # a 900-byte device, 100 reserved, every loaded context holding 400:
    # at most two systems at once (idle pooled contexts count as free)
    reqs = [_req(i, 0.0, steps=4, est=400) for i in range(6)]
    st = _loop(B, budget_bytes=10**9, reserve_bytes=100, make_context=make_ctx, load=load,
               free_memory=lambda dev: 900 - sum(c.device_bytes for c in live)).run(reqs)
    assert st.summary()["solves"] == 6
    assert 1 <= B.max_running <= 2


def test_contexts_are_pooled_and_closed():
    _Ctx.made = 0
    B = _Batch(0)
    reqs = [_req(i, 0.002 * i, steps=2) for i in range(12)]
    st = _loop(B, builders=2).run(reqs)
    assert st.summary()["solves"] == 12
    assert _Ctx.made < 12
