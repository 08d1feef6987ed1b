"""Host-side mirror of the reference's Simulation backend interface.

The reference selects a backend behind the abstract ``Simulation`` class
(src/Simulation/include/Simulation/Simulation.hpp:13-67): the UI thread calls
run() / pause() / set_timestep() / get_stats() / is_finished(), and the
backend advances the bodies on its own worker thread until ``iterations``
steps are done (src/Simulation/src/Simulation.cpp:33-72).  ``BarnesHutB200``
is that backend for the B200 library; ``NbContext`` is a thin owner of one
C-ABI context for callers that drive steps themselves (tests, benchmark).
"""
from __future__ import annotations

import ctypes as C
import enum
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import NbParams, NbStats, check, load, ptr


def _f64(a, shape) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64)
    if out.shape != shape:
        raise ValueError(f"expected shape {shape}, got {out.shape}")
    return out


@dataclass
class Bodies:
    """The reference's Bodies (src/common_lib/Body/include/Body/Body.hpp:10-40):
    ids, masses, interleaved positions and velocities, original order."""
    mass: np.ndarray
    pos: np.ndarray
    vel: np.ndarray
    ids: list[str] | None = None

    def __post_init__(self):
        n = int(np.asarray(self.mass).shape[0])
        self.mass = _f64(self.mass, (n,))
        self.pos = _f64(self.pos, (n, 2))
        self.vel = _f64(self.vel, (n, 2))
        if self.ids is None:
            self.ids = [str(i) for i in range(n)]

    @property
    def n(self) -> int:
        return int(self.mass.shape[0])


@dataclass
class SimConfig:
    """Config::Simulation (src/common_lib/Config/include/Config/Config.hpp:22-35)
    plus the values the reference fixes elsewhere: G (a compile-time constant
    in Constants.hpp:17) and the softening, passed directly as epsilon^2
    instead of being estimated from a random sample of pair distances
    (src/Simulation/src/Simulation.cpp:82-126)."""
    timestep: float = 1e-4
    iterations: int = 1000
    theta: float = 0.5
    epsilon_squared: float = 1e-4
    G: float = 1.0
    mode: int = _lib.NB_MODE_FP64
    leaf_size: int = 0
    device: int = 0
    quadrupole: bool = False
    learned: bool = False
    bmax_ratio: float = 0.0
    band_theta: float = 0.5  # learned mode: the plain walk's angle the network stands in for
    bodies_per_lane: int = 0  # SPLIT target groups of 32 x this (1, 2, 4; 0 = 1 below 131,072 bodies, else 2)
    cpu_law: bool = False   # NB_MODE_ALLPAIRS: the reference CPU backends' pair law

    def params(self) -> NbParams:
        p = NbParams()
        load().nb_params_default(C.byref(p))
        p.G = self.G
        p.timestep = self.timestep
        p.theta = self.theta
        p.epsilon_squared = self.epsilon_squared
        p.mode = self.mode
        p.leaf_size = self.leaf_size
        p.device = self.device
        p.bmax_ratio = self.bmax_ratio
        p.band_theta = self.band_theta
        p.bodies_per_lane = self.bodies_per_lane
        p.flags = ((_lib.NB_FLAG_QUADRUPOLE if self.quadrupole else 0)
                   | (_lib.NB_FLAG_LEARNED if self.learned else 0)
                   | (_lib.NB_FLAG_CPU_LAW if self.cpu_law else 0))
        return p


class NbContext:
    """Owns one nb_ctx of libnbody_b200.so."""

    def __init__(self, cfg: SimConfig, mass, pos, vel, counts=None):
        """counts (optional): bodies per universe for a batch of independent
        universes concatenated in mass/pos/vel (nb_batch_create)."""
        lib = load()
        self.cfg = cfg
        self._pending_upload = None
        self.n = int(np.asarray(mass).shape[0])
        mass = _f64(mass, (self.n,))
        pos = _f64(pos, (self.n, 2))
        vel = _f64(vel, (self.n, 2))
        h = C.c_void_p()
        p = cfg.params()
        if counts is None:
            check(lib.nb_create(C.byref(p), self.n, ptr(mass), ptr(pos), ptr(vel), C.byref(h)))
        else:
            cnt = np.ascontiguousarray(counts, dtype=np.uint64)
            if int(cnt.sum()) != self.n:
                raise ValueError("universe sizes must add up to the body count")
            check(lib.nb_batch_create(C.byref(p), cnt.shape[0], ptr(cnt), ptr(mass), ptr(pos),
                                      ptr(vel), C.byref(h)))
        self._h = h.value
        self._lib = lib

    # -- lifecycle --------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.nb_destroy(self._h)
            self._h = None
        self._pending_upload = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> int:
        if not self._h:
            raise RuntimeError("context is closed")
        return self._h

    # -- stepping ---------------------------------------------------------
    def step(self, nsteps: int = 1, sync: bool = True) -> None:
        check(self._lib.nb_step(self.handle, nsteps), self._h)
        if sync:
            self.sync()

    def sync(self) -> None:
        try:
            check(self._lib.nb_sync(self.handle), self._h)
        finally:
            self._pending_upload = None

    def set_timestep(self, dt: float) -> None:
        check(self._lib.nb_set_timestep(self.handle, dt), self._h)

    # -- data movement ----------------------------------------------------
    def upload(self, mass, pos, vel) -> None:
        mass = _f64(mass, (self.n,))
        pos = _f64(pos, (self.n, 2))
        vel = _f64(vel, (self.n, 2))
        check(self._lib.nb_upload(self.handle, ptr(mass), ptr(pos), ptr(vel)), self._h)

    def upload_async(self, mass: np.ndarray, pos: np.ndarray, vel: np.ndarray) -> None:
        """nb_upload_async: the copy overlaps the work enqueued before it; the
        arrays (pinned, C-contiguous float64 [n], [n, 2], [n, 2]) are read
        until sync() returns and are kept alive until then."""
        for a, shape in ((mass, (self.n,)), (pos, (self.n, 2)), (vel, (self.n, 2))):
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("upload_async needs C-contiguous float64 [n] / [n, 2] arrays")
        check(self._lib.nb_upload_async(self.handle, ptr(mass), ptr(pos), ptr(vel)), self._h)
        self._pending_upload = (mass, pos, vel)

    def download(self, pos: np.ndarray | None = None, vel: np.ndarray | None = None):
        if pos is None:
            pos = np.empty((self.n, 2))
        if vel is None:
            vel = np.empty((self.n, 2))
        check(self._lib.nb_download(self.handle, ptr(pos), ptr(vel)), self._h)
        return pos, vel

    def download_async(self, pos: np.ndarray, vel: np.ndarray) -> None:
        """nb_download_async: the copy overlaps what is enqueued next; pos and
        vel (pinned, [n, 2] float64) are valid after download_wait()."""
        for a in (pos, vel):
            if a.shape != (self.n, 2) or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("download_async needs C-contiguous float64 [n, 2] arrays")
        check(self._lib.nb_download_async(self.handle, ptr(pos), ptr(vel)), self._h)

    def download_wait(self) -> None:
        check(self._lib.nb_download_wait(self.handle), self._h)

    def accelerations(self) -> np.ndarray:
        acc = np.empty((self.n, 2))
        check(self._lib.nb_accelerations(self.handle, ptr(acc)), self._h)
        return acc

    # -- debug views ------------------------------------------------------
    def debug_morton(self):
        codes = np.empty(self.n, dtype=np.uint64)
        order = np.empty(self.n, dtype=np.int32)
        box = np.empty(4)
        check(self._lib.nb_debug_morton(self.handle, ptr(codes), ptr(order), ptr(box)), self._h)
        return codes, order, box

    def debug_state(self):
        mass = np.empty(self.n)
        pos = np.empty((self.n, 2))
        vel = np.empty((self.n, 2))
        orig = np.empty(self.n, dtype=np.int32)
        check(self._lib.nb_debug_state(self.handle, ptr(mass), ptr(pos), ptr(vel), ptr(orig)),
              self._h)
        return mass, pos, vel, orig

    def debug_tree(self):
        m = self.stats().tree_nodes
        cm = np.empty(max(m, 1))
        cc = np.empty((max(m, 1), 2))
        lv = np.empty(max(m, 1), dtype=np.int32)
        fb = np.empty(max(m, 1), dtype=np.int32)
        lb = np.empty(max(m, 1), dtype=np.int32)
        root = C.c_int32()
        check(self._lib.nb_debug_tree(self.handle, ptr(cm), ptr(cc), ptr(lv), ptr(fb), ptr(lb),
                                      C.addressof(root)), self._h)
        return dict(mass=cm[:m], com=cc[:m], level=lv[:m], first=fb[:m], last=lb[:m],
                    root=root.value)

    def debug_interactions(self):
        """FP64 mode: per-body (cell terms, body terms) of a force pass of the
        current state, in original order, and the deepest stack it used."""
        cells = np.empty(self.n, dtype=np.uint32)
        bodies = np.empty(self.n, dtype=np.uint32)
        hw = C.c_int32()
        check(self._lib.nb_debug_interactions(self.handle, ptr(cells), ptr(bodies),
                                              C.addressof(hw)), self._h)
        return cells, bodies, hw.value

    def debug_sort_passes(self, passes: int = -1) -> int:
        """The radix passes (top key bytes) the last sort took.  passes = 1..8
        forces that many for the following sorts, 0 returns to the automatic
        choice, -1 leaves the setting as it is."""
        last = C.c_int32()
        check(self._lib.nb_debug_sort_passes(self.handle, passes, C.addressof(last)), self._h)
        return last.value

    def debug_groups(self) -> np.ndarray:
        """SPLIT mode: [groups, 2] first and last body slot of each target group
        of the last step (device order)."""
        cnt = C.c_uint64()
        check(self._lib.nb_debug_groups(self.handle, None, None, 0, C.byref(cnt)), self._h)
        k = cnt.value
        first = np.empty(max(k, 1), dtype=np.int32)
        last = np.empty(max(k, 1), dtype=np.int32)
        check(self._lib.nb_debug_groups(self.handle, ptr(first), ptr(last), k, C.byref(cnt)),
              self._h)
        return np.stack([first[:k], last[:k]], axis=1)

    def phase_times(self) -> dict[str, float]:
        """Per-phase device ms of the last graph-launched step."""
        ms = np.zeros(16)
        k = self._lib.nb_phase_times(self.handle, ptr(ms), 16)
        if k < 0:
            check(-k, self._h)
        return {self._lib.nb_phase_name(i).decode(): float(ms[i]) for i in range(k)}

    def render(self, view, point_diameter: float = 1.0) -> np.ndarray:
        """The current bodies drawn as the reference's window would show them
        (nb_render): view is a render.ViewPort or an NbView; returns
        [res_y, res_x, 4] uint8, row 0 at the top."""
        v = view.as_view(point_diameter) if hasattr(view, "as_view") else view
        out = np.empty((v.res_y, v.res_x, 4), dtype=np.uint8)
        check(self._lib.nb_render(self.handle, C.byref(v), out.ctypes.data), self._h)
        return out

    def autotune(self, steps: int = 3) -> tuple[int, int]:
        """Times the SPLIT leaf sizes and group sizes; returns (leaf, bodies per lane)."""
        leaf, bpl = C.c_int32(), C.c_int32()
        check(self._lib.nb_autotune(self.handle, steps, C.addressof(leaf), C.addressof(bpl)),
              self._h)
        return leaf.value, bpl.value

    # -- learned correction -----------------------------------------------
    def set_mlp_weights(self, params: np.ndarray) -> None:
        params = np.ascontiguousarray(params, dtype=np.float32)
        if params.shape != (_lib.NB_MLP_PARAMS,):
            raise ValueError(f"expected {_lib.NB_MLP_PARAMS} parameters")
        check(self._lib.nb_set_mlp_weights(self.handle, ptr(params)), self._h)

    def mlp_samples(self, ntargets: int, seed: int = 0, capacity: int | None = None):
        """Residual samples (features[k,12], residuals[k,2]) of the current bodies,
        from `ntargets` random target groups."""
        capacity = capacity or 256 * ntargets
        X = np.empty((capacity, 12), dtype=np.float32)
        Y = np.empty((capacity, 2), dtype=np.float32)
        cnt = C.c_uint64()
        check(self._lib.nb_mlp_samples(self.handle, ntargets, seed, capacity, ptr(X), ptr(Y),
                                       C.byref(cnt)), self._h)
        return X[:cnt.value], Y[:cnt.value]

    def stats(self) -> NbStats:
        s = NbStats()
        check(self._lib.nb_get_stats(self.handle, C.byref(s)), self._h)
        return s


def allpairs_accelerations(mass, pos, targets, epsilon_squared: float, device: int = 0) -> np.ndarray:
    """FP64 all-pairs accelerations of the given targets on the GPU."""
    lib = load()
    n = int(np.asarray(mass).shape[0])
    mass = _f64(mass, (n,))
    pos = _f64(pos, (n, 2))
    tgt = np.ascontiguousarray(targets, dtype=np.int64)
    acc = np.empty((tgt.shape[0], 2))
    check(lib.nb_allpairs_accelerations(device, n, ptr(mass), ptr(pos), tgt.shape[0], ptr(tgt),
                                        epsilon_squared, ptr(acc)))
    return acc


def mlp_forward(params, features, device: int = 0) -> np.ndarray:
    """Raw network outputs [n, 2] (without the output scale) on the GPU."""
    lib = load()
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(features, dtype=np.float32)
    out = np.empty((X.shape[0], 2), dtype=np.float32)
    check(lib.nb_mlp_forward(device, ptr(params), X.shape[0], ptr(X), ptr(out)))
    return out


def mlp_loss_grad(params, features, targets, device: int = 0):
    """(mean squared error, gradient[NB_MLP_PARAMS]) on the GPU."""
    lib = load()
    params = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(features, dtype=np.float32)
    T = np.ascontiguousarray(targets, dtype=np.float32)
    grad = np.empty(_lib.NB_MLP_PARAMS, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    check(lib.nb_mlp_loss_grad(device, ptr(params), X.shape[0], ptr(X), ptr(T), ptr(grad),
                               ptr(loss)))
    return float(loss[0]), grad


def mlp_train(features, residuals, *, epochs: int = 4, batch: int = 4096, lr: float = 2e-3,
              seed: int = 0, params=None, device: int = 0):
    """Trains the correction MLP on the GPU; returns (params, loss per epoch)."""
    lib = load()
    X = np.ascontiguousarray(features, dtype=np.float32)
    Y = np.ascontiguousarray(residuals, dtype=np.float32)
    P = (np.zeros(_lib.NB_MLP_PARAMS, dtype=np.float32) if params is None
         else np.array(params, dtype=np.float32))
    losses = np.zeros(epochs, dtype=np.float32)
    tp = _lib.NbMlpTrainParams(epochs=epochs, batch=batch, lr=lr, seed=seed)
    check(lib.nb_mlp_train(device, X.shape[0], ptr(X), ptr(Y), C.byref(tp), ptr(P), ptr(losses)))
    return P, losses


class State(enum.Enum):
    PAUSED = 0
    RUNNING = 1


@dataclass
class Stats:
    """Simulation::Stats (Simulation.hpp:17-22)."""
    iteration: int = 0
    ips: float = 0.0
    real_elapsed_s: float = 0.0
    simulated_elapsed_s: float = 0.0


class Simulation:
    """Mirror of the reference's abstract Simulation (Simulation.hpp:13-67):
    run/pause state under a lock, a stop flag, an iteration cap, a timestep
    hot-swap applied between steps, and rate-limited stats."""

    STATS_MIN_INTERVAL_S = 50e-6  # Constants::Simulation::STATS_UPDATE_TIMER

    def __init__(self, cfg: SimConfig, bodies: Bodies):
        self.cfg = cfg
        self.bodies = bodies
        self.timestep = cfg.timestep
        self.max_iterations = cfg.iterations
        self.iteration = 0
        self._requested_timestep = cfg.timestep
        self._state = State.PAUSED
        self._state_mtx = threading.Lock()
        self._stats_mtx = threading.Lock()
        self._stats = Stats()
        self._finished = threading.Event()
        self._stop = threading.Event()
        self._elapsed = 0.0
        self._resumed_at: float | None = None
        self._last_stats_call = 0.0
        self._ips_samples: list[float] = []

    # Simulation.cpp:33-42
    def run(self) -> None:
        with self._state_mtx:
            if self._state != State.PAUSED:
                return
            self._state = State.RUNNING
            self.on_run()
            self._resumed_at = time.perf_counter()

    # Simulation.cpp:44-53
    def pause(self) -> None:
        with self._state_mtx:
            if self._state != State.RUNNING:
                return
            self._state = State.PAUSED
            self.on_pause()
            if self._resumed_at is not None:
                self._elapsed += time.perf_counter() - self._resumed_at
                self._resumed_at = None

    def get_state(self) -> State:
        with self._state_mtx:
            return self._state

    def get_stats(self) -> Stats:
        with self._stats_mtx:
            return Stats(**vars(self._stats))

    def is_finished(self) -> bool:
        return self._finished.is_set()

    def set_timestep(self, dt: float) -> None:
        self._requested_timestep = float(dt)

    # Simulation.cpp:59-72
    def should_stop(self) -> bool:
        if self.iteration >= self.max_iterations:
            self._finished.set()
            return True
        return self._stop.is_set()

    def post_iteration(self, iterations: int = 1) -> None:
        now = time.perf_counter()
        if now - self._last_stats_call >= self.STATS_MIN_INTERVAL_S:
            self._last_stats_call = now
            self._update_stats(iterations)
        self.timestep = self._requested_timestep
        self.iteration += iterations

    def _update_stats(self, iterations: int) -> None:
        elapsed = self._elapsed + (time.perf_counter() - self._resumed_at
                                   if self._resumed_at is not None else 0.0)
        with self._stats_mtx:
            d_it = self.iteration + iterations - self._stats.iteration
            dt = elapsed - self._stats.real_elapsed_s
            if dt > 0:
                self._ips_samples = (self._ips_samples + [d_it / dt])[-60:]
                self._stats.ips = float(np.mean(self._ips_samples))
            self._stats.iteration = self.iteration + iterations
            self._stats.real_elapsed_s = elapsed
            self._stats.simulated_elapsed_s += d_it * self.timestep

    def on_run(self) -> None:  # pragma: no cover - abstract
        raise NotImplementedError

    def on_pause(self) -> None:  # pragma: no cover - abstract
        raise NotImplementedError


class BarnesHutB200(Simulation):
    """The B200 backend (stands in for BarnesHutCuda,
    src/Simulation/src/BarnesHutCuda.cpp:1-40).  ``download_every`` = 1
    copies the bodies back after every step as the reference does
    (BarnesHutCuda.cu:632-646); larger values keep the state on the GPU and
    copy it back every that many steps and when paused or finished."""

    def __init__(self, cfg: SimConfig, bodies: Bodies, download_every: int = 1):
        super().__init__(cfg, bodies)
        self.download_every = max(1, int(download_every))
        self.ctx = NbContext(cfg, bodies.mass, bodies.pos, bodies.vel)
        self._thread: threading.Thread | None = None
        self.error: Exception | None = None

    def on_run(self) -> None:
        self._stop.clear()
        self._thread = threading.Thread(target=self._simulate, daemon=True)
        self._thread.start()

    def on_pause(self) -> None:
        self._stop.set()
        if self._thread is not None:
            self._thread.join()
            self._thread = None

    def _simulate(self) -> None:
        try:
            while not self.should_stop():
                if self.timestep != self.ctx.cfg.timestep:
                    self.ctx.set_timestep(self.timestep)
                    self.ctx.cfg.timestep = self.timestep
                k = min(self.download_every, self.max_iterations - self.iteration)
                self.ctx.step(k, sync=True)
                self.ctx.download(self.bodies.pos, self.bodies.vel)
                self.post_iteration(k)
            self.ctx.download(self.bodies.pos, self.bodies.vel)
        except Exception as exc:  # the C++ adapter logs and stops; so do we
            self.error = exc
            self._finished.set()

    def close(self) -> None:
        if self.get_state() == State.RUNNING:
            self.pause()
        self.ctx.close()
