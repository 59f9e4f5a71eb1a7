"""The multi-GPU request router (one solve server per device) on fake
servers: requests go to the device with the least outstanding cells x steps
among those whose budget holds them; finished and cancelled requests leave the
account; the load over a Poisson stream of the serving configuration stays
even."""
import numpy as np
import pytest

from acoustics_b200 import scene as S
from acoustics_b200.router import ServerRouter, balance


class FakeServer:
    def __init__(self, device, precision, hbm_budget_bytes, **kw):
        self.device = device
        self.next = 1
        self.live = {}
        self.cancelled = []

    def submit(self, scene, steps):
        rid = self.next
        self.next += 1
        self.live[rid] = (scene, steps)
        return rid

    def result(self, rid):
        scene, steps = self.live.pop(rid)
        return np.zeros((steps, scene.n_listeners)), 0.0

    def cancel(self, rid):
        self.live.pop(rid)
        self.cancelled.append(rid)

    def stats(self):
        return {"running": len(self.live)}

    def close(self):
        pass


def scene(n, steps=100):
    return S.Scene(cell_size=0.005, divisions=(n, n, n), time_step=1e-6, steps=steps, name=f"s{n}")


def make(budget=0, devices=(0, 1, 2, 3)):
    return ServerRouter(devices=devices, hbm_budget_bytes=budget, server_factory=FakeServer,
                        footprint=lambda sc: sc.n_cells * 100)


def test_least_outstanding_work_first():
    r = make()
    k1 = r.submit(scene(100))          # -> 0
    k2 = r.submit(scene(50))           # -> 1
    k3 = r.submit(scene(50))           # -> 2
    k4 = r.submit(scene(50))           # -> 3
    k5 = r.submit(scene(40))           # -> 1 (ties with 2 and 3 broken by index; 0 holds the most)
    assert [k[0] for k in (k1, k2, k3, k4, k5)] == [0, 1, 2, 3, 1]
    r.result(k1)                       # device 0 is empty again
    assert r.submit(scene(40))[0] == 0
    r.cancel(k2)
    assert r.work[1] == pytest.approx(40 ** 3 * 100)
    assert r.servers[1].cancelled == [k2[1]]


def test_budget_decides_where_a_request_fits():
    r = make(budget=10 ** 8)
    big = scene(100)                   # 1e8 bytes: fits exactly
    assert r.submit(big)[0] == 0
    with pytest.raises(ValueError):
        r.submit(scene(120))           # 1.7e8 bytes: fits nowhere


def test_even_load_on_a_poisson_stream():
    r = make()
    for _, sc in S.config4(n_requests=64, rate_per_s=16.0):
        r.submit(sc)
    assert balance(r.work) < 1.25
    assert sum(r.counts) == 64 and min(r.counts) >= 8
