"""Host-side logic without a GPU: the Simulation mirror's run/pause/iteration
cap/timestep hot-swap/stats (src/Simulation/src/Simulation.cpp:33-72), the
universe generators, and the benchmark's replica reduction under two gloo
ranks (the step does not shard: replicas only)."""
import os
import threading
import time

import numpy as np
import pytest


class FakeBackend:
    """Stands in for the B200 library: counts steps and records timesteps."""

    def __init__(self):
        self.steps = 0
        self.dts = []


def make_sim(nbp, iterations, fake):
    class FakeSim(nbp.Simulation):
        def on_run(self):
            self._stop.clear()
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()

        def on_pause(self):
            self._stop.set()
            self._thread.join()

        def _loop(self):
            while not self.should_stop():
                fake.steps += 1
                fake.dts.append(self.timestep)
                time.sleep(0.0005)
                self.post_iteration()

    b = nbp.Bodies(np.ones(3), np.zeros((3, 2)), np.zeros((3, 2)))
    return FakeSim(nbp.SimConfig(timestep=1e-3, iterations=iterations), b)


def test_run_until_iteration_cap(nbp):
    fake = FakeBackend()
    sim = make_sim(nbp, 25, fake)
    assert sim.get_state() == nbp.State.PAUSED
    sim.run()
    for _ in range(2000):
        if sim.is_finished():
            break
        time.sleep(0.001)
    assert sim.is_finished() and fake.steps == 25
    sim.pause()
    st = sim.get_stats()
    assert 0 < st.iteration <= 25 and st.simulated_elapsed_s > 0


def test_pause_resume_and_timestep_hot_swap(nbp):
    fake = FakeBackend()
    sim = make_sim(nbp, 10 ** 9, fake)
    sim.run()
    sim.run()  # a second run while running is ignored, as in Simulation::run
    time.sleep(0.02)
    sim.set_timestep(2e-3)
    time.sleep(0.02)
    sim.pause()
    n1 = fake.steps
    time.sleep(0.01)
    assert fake.steps == n1  # paused: no progress
    assert fake.dts[0] == 1e-3 and fake.dts[-1] == 2e-3
    sim.run()
    time.sleep(0.01)
    sim.pause()
    assert fake.steps > n1


def test_universe_generators(nbp):
    u = nbp.universes
    m, p, v = u.exponential_disc(1000, 0)
    assert m[0] == pytest.approx(1e5 * m[1]) and m[1:].sum() == pytest.approx(1.0)
    r = np.linalg.norm(p[1:], axis=1)
    assert r.max() <= 10.0 and abs(np.median(r) - np.log(2)) < 0.1
    m2, p2, v2 = u.colliding_discs(2000, 0)
    assert m2.shape == (2000,) and abs(p2[:1000, 0].mean() + 20) < 1 and abs(p2[1000:, 0].mean() - 20) < 1
    # the central bodies sit at x = -+20 and carry the discs' bulk velocities
    assert p2[0].tolist() == [-20.0, 0.0] and p2[1000].tolist() == [20.0, 0.0]
    assert v2[0].tolist() == [0.0, 0.25] and v2[1000].tolist() == [0.0, -0.25]
    m3, p3, v3 = u.plummer_disc(5000, 1)
    assert m3.sum() == pytest.approx(1.0) and abs(v3.std() - 0.3) < 0.02
    sizes = u.ensemble_sizes(512, 0)
    assert sizes.min() >= 1024 and sizes.max() <= 262144
    assert np.array_equal(u.exponential_disc(100, 7)[1], u.exponential_disc(100, 7)[1])


def _replica_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    ms = 1.0 + rank  # rank 1 is the slow one
    q.put((rank, bench.max_over_ranks(ms)))
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(120)
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 2.0, 1: 2.0}
