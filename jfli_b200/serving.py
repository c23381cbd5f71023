"""Continuous-batching engine for forward-model requests (sampler chains asking for
density + P(k) at a cosmology and a white-noise seed).

Requests are grouped by mesh size. Each size owns a fixed set of slots whose particle
state, density, force meshes and FFT workspace stay resident on the GPU (the slot count
per size comes from the HBM budget). Every engine tick advances all active slots of a
size by one PM step with a single batched step (`jfli_pm_step_slots`), each slot with its
own kick/drift factors (its own cosmology, step count and position in its schedule).
The step's launches are recorded once per size as a CUDA graph and replayed; per-slot
factors are copied to device arrays before each replay. A request that arrives while
others are running waits for a free slot of its size, is then set up (ICs, 2LPT, first
force) into that slot and joins the next tick, so its work overlaps the others' on the
device. A finished slot's density is painted by its last step; P(k) and the host copy
are enqueued and the slot is reused at once.

Host-side preparation (cosmology tables, LPT factors, the KDK schedule) runs in a pool
of spawned worker processes so it overlaps the GPU work.

The reference's request source is `make_full_field_model` (probabilistic_models/
forward_model.py:24-79) called from the samplers in infer/batched_sampling.py; one
request here is one forward evaluation of that model's lpt -> nbody -> power chain.
"""

from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import math
import multiprocessing as mp
import time
from collections import deque

import numpy as np
import torch

from . import _lib, ops
from ._lib import JFLI_STEP_CLEAR, JFLI_STEP_DRIFT, JFLI_STEP_KICK, JFLI_STEP_PAINT

A_INIT = 0.1


@dataclasses.dataclass
class ForwardRequest:
    rid: int
    mesh: int
    box: float
    omega_c: float
    sigma8: float
    steps: int
    seed: int
    want_grad: bool = False
    arrival: float = 0.0  # seconds after the stream starts


@dataclasses.dataclass
class ForwardResult:
    rid: int
    density: torch.Tensor  # host (pinned) copy of the final CIC density
    k: np.ndarray
    pk: np.ndarray
    steps: int
    arrival: float
    admitted: float = 0.0
    done: float = 0.0
    # gradient requests: loss and gradients of the log-P(k) loss (reversible adjoint)
    loss: float | None = None
    grad_noise: torch.Tensor | None = None  # host copy, (mesh,)*3
    grad_omega_c: float | None = None
    grad_sigma8: float | None = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def config_kedges(n: int, box: float) -> np.ndarray:
    """33 log-spaced edges from the fundamental to the Nyquist wavenumber (32 bins)."""
    return np.geomspace(2 * np.pi / box * (1 - 1e-6), np.pi * n / box, 33)


def prepare(req: ForwardRequest) -> dict:
    """Host-side FP64 tables of one request (runs in a worker process)."""
    from . import cosmology as cj
    from .pm.integrate import time_events
    from .pm.lpt import lpt_coefficients
    from .pm.solvers import EfficientDriftDoubleKick as EDK

    c = cj.Planck18(Omega_c=float(req.omega_c), sigma8=float(req.sigma8))
    k, pk = cj.pk_table(c, 128)
    dt0 = (1.0 - A_INIT) / req.steps
    ev = [(e[1], e[2]) for e in time_events(A_INIT, [1.0], dt0) if e[0] == "step"]
    kicks, drifts = EDK.schedule_arrays(c, [a for a, _ in ev], [b for _, b in ev], dt0)
    out = dict(rid=req.rid, ktab=k.astype(np.float32), ptab=pk.astype(np.float32),
               lpt=lpt_coefficients(c, A_INIT), init_kick=EDK.init_kick(c, A_INIT, A_INIT + dt0),
               kicks=np.asarray(kicks, np.float64), drifts=np.asarray(drifts, np.float64),
               kedges=config_kedges(req.mesh, req.box).astype(np.float32))
    if req.want_grad:
        from .pm.adjoint import forward_tables

        out["grad_tables"] = forward_tables(req.omega_c, req.sigma8, t0=A_INIT, t1=1.0, dt0=dt0)
    return out


# Target spectrum of the gradient requests' loss: the fiducial cosmology, a second seed.
TARGET_SEED = 1_000_003
FIDUCIAL = (0.2607, 0.8102)


def gradient_request(req: ForwardRequest, prep: dict, pk_target: torch.Tensor):
    """Loss sum_b (log P_b - log P_target,b)^2 of the request's ReversibleDoubleKickDrift
    run (its mesh, cosmology and step count) and its gradients with respect to the white
    noise, Omega_c and sigma8 through the reversible adjoint. Enqueued on the current stream."""
    from .pm.adjoint import forward_model_pk, pk_log_loss

    w = device_white_noise(req.seed, req.mesh).requires_grad_(True)
    om = torch.tensor(float(req.omega_c), dtype=torch.float64, requires_grad=True)
    sg = torch.tensor(float(req.sigma8), dtype=torch.float64, requires_grad=True)
    pk = forward_model_pk(w, om, sg, box=(req.box,) * 3, kedges=config_kedges(req.mesh, req.box), t0=A_INIT,
                          dt0=(1.0 - A_INIT) / req.steps, tables=prep["grad_tables"])
    loss = pk_log_loss(pk, pk_target)
    loss.backward()
    return loss.detach(), w.grad, om.grad, sg.grad


def target_spectrum(n: int, box: float, steps: int = 20) -> torch.Tensor:
    from .pm.adjoint import forward_model_pk

    with torch.no_grad():
        return forward_model_pk(device_white_noise(TARGET_SEED, n), torch.tensor(FIDUCIAL[0]),
                                torch.tensor(FIDUCIAL[1]), box=(box,) * 3, kedges=config_kedges(n, box), t0=A_INIT,
                                dt0=(1.0 - A_INIT) / steps)


class GradientWorker:
    """Runs gradient requests from host threads, each thread on its own CUDA stream, so
    that they run concurrently with the batched forward steps on the main stream and,
    for small meshes that do not fill the GPU, with one another."""

    def __init__(self, threads: int = 3):
        import queue
        import threading

        self.inbox: "queue.Queue" = queue.Queue()
        self.outbox: "queue.Queue" = queue.Queue()
        self.targets: dict = {}
        self.streams = [torch.cuda.Stream() for _ in range(max(1, threads))]
        self.t0 = time.perf_counter()
        self._threads = [threading.Thread(target=self._loop, args=(st,), daemon=True) for st in self.streams]
        for t in self._threads:
            t.start()

    def target(self, n: int, box: float) -> torch.Tensor:
        """Target spectrum of a mesh size (built once, before requests of that size run)."""
        key = (n, box)
        if key not in self.targets:
            st = self.streams[0]
            with torch.cuda.stream(st):
                spec = target_spectrum(n, box)
            st.synchronize()
            self.targets[key] = spec
        return self.targets[key]

    def submit(self, req, prep):
        self.inbox.put((req, prep))

    def _loop(self, stream):
        while True:
            item = self.inbox.get()
            if item is None:
                return
            req, prep = item
            try:
                with torch.cuda.stream(stream):
                    loss, gw, gom, gs8 = gradient_request(req, prep, self.targets[(req.mesh, req.box)])
                    gw_h = torch.empty(gw.shape, dtype=torch.float32, pin_memory=True)
                    gw_h.copy_(gw, non_blocking=True)
                stream.synchronize()
                self.outbox.put((req.rid, float(loss), gw_h, float(gom), float(gs8), time.perf_counter(), None))
            except Exception as exc:  # reported to the caller through the outbox
                self.outbox.put((req.rid, None, None, None, None, time.perf_counter(), exc))

    def close(self):
        for _ in self._threads:
            self.inbox.put(None)
        for t in self._threads:
            t.join(timeout=60)


def device_white_noise(seed: int, n: int, device="cuda") -> torch.Tensor:
    """N(0, 1) white noise of one request, generated on the device from its seed."""
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return torch.randn((n, n, n), generator=g, device=device, dtype=torch.float32)


def _pinned_to_device(arr: np.ndarray) -> torch.Tensor:
    """Host array -> device tensor without blocking the host (pinned staging copy)."""
    return torch.from_numpy(np.ascontiguousarray(arr)).pin_memory().to("cuda", non_blocking=True)


def setup_request(req: ForwardRequest, prep: dict, x_out: torch.Tensor, v_out: torch.Tensor):
    """ICs and 2LPT of one request written into (x_out, v_out); enqueued without a host sync."""
    n = req.mesh
    noise = device_white_noise(req.seed, n)
    ktab = _pinned_to_device(prep["ktab"])
    ptab = _pinned_to_device(prep["ptab"])
    ic = ops.ic_filter(noise, ktab, ptab, (req.box,) * 3)
    ops.lpt(ic, 2, *prep["lpt"], dx=x_out, p=v_out)


class _Slot:
    __slots__ = ("req", "prep", "idx", "pending", "admitted")

    def __init__(self, req, prep, admitted):
        self.req = req
        self.prep = prep
        self.idx = 0
        self.pending = prep["init_kick"]
        self.admitted = admitted


class SizeGroup:
    """All slots of one mesh size: resident state, the batched step and its CUDA graphs.

    Active slots are kept packed in indices 0..n_active-1 (a finished slot's index is
    refilled by moving the last active slot's particles and force meshes into it), so one
    batched step over the first n_active slots advances every request of this size and no
    work is spent on idle slots. One graph per active count is recorded up front.

    The per-slot step parameters (kick, drift, flags) live in one (3, B) device array
    that the graphs read. Each tick fills a pinned host buffer from a small ring and
    copies it over; a buffer is reused only after the event recorded behind its copy has
    completed, so the host can run ahead of the device without overwriting parameters
    that are still in flight."""

    RING = 8

    def __init__(self, n: int, capacity: int, use_graph: bool = True):
        self.n = n
        self.B = capacity
        dev = "cuda"
        self.x = torch.zeros(capacity, n, n, n, 3, device=dev)
        self.v = torch.zeros_like(self.x)
        self.rho = torch.zeros(capacity, n, n, n, device=dev)
        self.force = torch.zeros(capacity, n, n, n, 4, device=dev)
        self.pot1 = torch.empty(n, n, n, device=dev)
        nb = _lib.query("jfli_pm_step_workspace_bytes", n, n, n, capacity)
        self.ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        # rows: kick (f32 bits), drift (f32 bits), flags (i32)
        self.params_d = torch.zeros(3, capacity, dtype=torch.int32, device=dev)
        self._ring_h = [torch.zeros(3, capacity, dtype=torch.int32).pin_memory() for _ in range(self.RING)]
        self._ring_np = [h.numpy() for h in self._ring_h]
        self._ring_ev = [None] * self.RING
        self._ring_i = 0
        self.slots: list[_Slot] = []  # active slots, packed
        self.use_graph = use_graph
        self.graphs: dict[int, torch.cuda.CUDAGraph] = {}
        self._kedges: dict[float, torch.Tensor] = {}
        self.ticks = 0

    @staticmethod
    def bytes_per_slot(n: int) -> int:
        # x, v (24 B) + density (4) + force mesh (16) + half spectrum and potential (~8 B per cell)
        return int(52 * n**3 + 8 * n * n * (n // 2 + 1))

    def has_room(self) -> bool:
        return len(self.slots) < self.B

    def n_active(self) -> int:
        return len(self.slots)

    def _launch(self, nb: int):
        n, B = self.n, self.B
        base = self.params_d.data_ptr()
        _lib.call("jfli_pm_step_slots", _lib.stream_ptr(), _lib.ptr(self.x), _lib.ptr(self.v), base, base + 4 * B,
                  base + 8 * B, _lib.ptr(self.rho), _lib.ptr(self.force), _lib.ptr(self.ws), self.ws.numel(), n, n,
                  n, nb)

    def prepare_graphs(self):
        """Record the batched step for every active count 1..B. Must run while no slot is
        active: the eager run that precedes the captures (it creates the FFT tables and
        sets kernel attributes) overwrites the density and force meshes of every slot."""
        if self.slots:
            raise RuntimeError("prepare_graphs needs an idle group")
        self.params_d.zero_()
        self._launch(self.B)
        torch.cuda.synchronize()
        if self.use_graph:
            for nb in range(1, self.B + 1):
                if nb not in self.graphs:
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, capture_error_mode="thread_local"):
                        self._launch(nb)
                    self.graphs[nb] = g

    def kedges(self, prep: dict, box: float) -> torch.Tensor:
        t = self._kedges.get(box)
        if t is None:
            t = _pinned_to_device(prep["kedges"])
            self._kedges[box] = t
        return t

    def admit(self, req: ForwardRequest, prep: dict, now: float) -> int:
        b = len(self.slots)
        setup_request(req, prep, self.x[b], self.v[b])
        # force at the slot's initial positions
        ops.kick_drift_paint(self.x[b], self.v[b], None, 0.0, 0.0, JFLI_STEP_PAINT | JFLI_STEP_CLEAR, self.rho[b])
        ops.poisson_force(self.rho[b], 1.0, out=self.force[b], pot=self.pot1)
        self.slots.append(_Slot(req, prep, now))
        return b

    def release(self, b: int):
        """Free slot b (its results already enqueued): the last active slot moves into b."""
        last = len(self.slots) - 1
        if b != last:
            self.x[b].copy_(self.x[last])
            self.v[b].copy_(self.v[last])
            self.force[b].copy_(self.force[last])
            self.slots[b] = self.slots[last]
        self.slots.pop()

    def tick(self):
        """One PM step for every active slot; returns the indices whose schedule ended
        (descending, the order in which they can be finalized and released)."""
        nb = len(self.slots)
        r = self._ring_i
        self._ring_i = (r + 1) % self.RING
        if self._ring_ev[r] is not None:
            self._ring_ev[r].synchronize()
        h = self._ring_np[r]
        kick = h[0].view(np.float32)
        drift = h[1].view(np.float32)
        flags = h[2]
        step_flags = JFLI_STEP_KICK | JFLI_STEP_DRIFT | JFLI_STEP_PAINT
        for b, s in enumerate(self.slots):
            kick[b] = s.pending
            drift[b] = s.prep["drifts"][s.idx]
            flags[b] = step_flags
        self.params_d.copy_(self._ring_h[r], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self._ring_ev[r] = ev
        g = self.graphs.get(nb)
        if g is not None:
            g.replay()
        else:
            self._launch(nb)
        self.ticks += 1
        finished = []
        for b, s in enumerate(self.slots):
            s.pending = s.prep["kicks"][s.idx]
            s.idx += 1
            if s.idx == len(s.prep["kicks"]):
                finished.append(b)
        return finished[::-1]


def slot_capacities(sizes, hbm_budget_gb: float, max_slots: int) -> dict:
    """Slots per mesh size: an equal share of the HBM budget each, at least 1, at most max_slots."""
    share = hbm_budget_gb * 1e9 / len(sizes)
    return {int(n): int(max(1, min(max_slots, share // SizeGroup.bytes_per_slot(int(n))))) for n in sizes}


class Engine:
    """Admission by HBM budget, continuous batching per mesh size, CUDA-graph replay."""

    def __init__(self, sizes=(64, 96, 128, 192), hbm_budget_gb: float = 24.0, max_slots: int = 16,
                 use_graph: bool = True, workers: int = 6, keep_density: bool | str = True, grad_threads: int = 3,
                 on_result=None):
        """keep_density: True returns each density in pinned host memory, "device" as a
        CUDA tensor of the caller's own, False not at all (P(k) only).
        on_result(res): called once per request as soon as its result is complete (the
        density and P(k) ready to use), before it is stored in `results`; a consumer that
        takes the density and sets `res.density = None` lets its memory be reused."""
        self.groups: dict[int, SizeGroup] = {}
        for n, cap in slot_capacities(sizes, hbm_budget_gb, max_slots).items():
            self.groups[n] = SizeGroup(n, cap, use_graph=use_graph)
        self.workers = workers
        self.keep_density = keep_density
        self.grad_threads = grad_threads
        self.on_result = on_result
        self._pool = None
        self._ready = False
        self.results: dict[int, ForwardResult] = {}
        self._inflight = []  # finished slots whose P(k) / density copies are still on the stream
        self._grad = None
        self._await_grad: dict[int, ForwardResult] = {}  # forward done, gradient pending
        self._grad_done: dict[int, tuple] = {}  # gradient done, forward pending
        # host seconds of the serving loop by phase (admit: ICs + 2LPT + first force enqueued;
        # tick: batched step launches; finalize: P(k) and copies enqueued; poll: results
        # collected; idle: waits for the GPU, for arrivals or for gradients) and the number
        # of loop passes in which an arrived request waited for its host tables
        self.stats = dict(admit_s=0.0, tick_s=0.0, finalize_s=0.0, poll_s=0.0, idle_s=0.0, prep_waits=0,
                          loop_passes=0)

    def capacity(self) -> dict:
        return {n: g.B for n, g in self.groups.items()}

    def warmup(self):
        """Start the host workers and record every group's step graph (all slots idle)."""
        if self.workers > 0 and self._pool is None:
            self._pool = cf.ProcessPoolExecutor(self.workers, mp_context=mp.get_context("spawn"))
            probe = ForwardRequest(rid=-1, mesh=64, box=256.0, omega_c=0.26, sigma8=0.81, steps=10, seed=0)
            for f in [self._pool.submit(prepare, probe) for _ in range(self.workers)]:
                f.result()
        if not self._ready:
            for g in self.groups.values():
                g.prepare_graphs()
            self._ready = True

    def close(self):
        if self._pool is not None:
            self._pool.shutdown(wait=True, cancel_futures=True)
            self._pool = None
        if self._grad is not None:
            self._grad.close()
            self._grad = None

    def _gradient_worker(self) -> GradientWorker:
        if self._grad is None:
            self._grad = GradientWorker(self.grad_threads)
        return self._grad

    def _finalize(self, g: SizeGroup, b: int):
        s = g.slots[b]
        req = s.req
        sums = ops.power_sums(g.rho[b], g.kedges(s.prep, req.box), (req.box,) * 3)
        dens = None
        if self.keep_density == "device":
            dens = g.rho[b].clone()  # the caller's own copy on the GPU (the slot is reused at once)
        elif self.keep_density:
            dens = torch.empty(req.mesh, req.mesh, req.mesh, dtype=torch.float32, pin_memory=True)
            dens.copy_(g.rho[b], non_blocking=True)
        sums_h = torch.empty(sums.shape, dtype=torch.float64, pin_memory=True)
        sums_h.copy_(sums, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        res = ForwardResult(rid=req.rid, density=dens, k=None, pk=None, steps=len(s.prep["kicks"]),
                            arrival=req.arrival, admitted=s.admitted)
        self._inflight.append((ev, res, sums_h, req))
        g.release(b)

    def _poll(self, now_fn):
        keep = []
        for item in self._inflight:
            ev, res, sums_h, req = item
            if not ev.query():
                keep.append(item)
                continue
            s = sums_h.numpy()
            cnt = np.where(s[1] > 0, s[1], 1.0)
            vol = (req.box / req.mesh) ** 3
            res.pk = (s[0] / cnt)[1:-1] * vol
            res.k = (s[2] / cnt)[1:-1]
            res.done = now_fn()
            if req.want_grad:
                self._await_grad[res.rid] = res
            else:
                self._deliver(res)
        self._inflight = keep
        if self._grad is not None:
            while not self._grad.outbox.empty():
                rid, loss, gw, gom, gs8, t_done, exc = self._grad.outbox.get()
                if exc is not None:
                    raise RuntimeError(f"gradient request {rid} failed") from exc
                self._grad_done[rid] = (loss, gw, gom, gs8, t_done - self._t0_abs)
        for rid in [r for r in self._await_grad if r in self._grad_done]:
            res = self._await_grad.pop(rid)
            loss, gw, gom, gs8, t_done = self._grad_done.pop(rid)
            res.loss, res.grad_noise, res.grad_omega_c, res.grad_sigma8 = loss, gw, gom, gs8
            res.done = max(res.done, t_done)
            self._deliver(res)

    def _deliver(self, res):
        if self.on_result is not None:
            self.on_result(res)
        self.results[res.rid] = res

    def run(self, requests, realtime: bool = True):
        """Serve `requests` (arrival times in seconds after the call); returns {rid: ForwardResult}.
        Request ids must be unique, and new to this engine (results are keyed by id)."""
        rids = [r.rid for r in requests]
        if len(set(rids)) != len(rids):
            raise ValueError("request ids must be unique within a run")
        seen = [rid for rid in rids if rid in self.results]
        if seen:
            raise ValueError(f"request ids already served by this engine: {seen[:8]}")
        for r in requests:
            if r.mesh not in self.groups:
                raise ValueError(f"request {r.rid}: mesh {r.mesh} has no slot group (sizes {list(self.groups)})")
        self.warmup()
        pool = self._pool
        reqs = sorted(requests, key=lambda r: r.arrival)
        if any(r.want_grad for r in reqs):
            gw = self._gradient_worker()
            for key in sorted({(r.mesh, r.box) for r in reqs if r.want_grad}):
                gw.target(*key)
        t0 = time.perf_counter()
        self._t0_abs = t0
        now = lambda: time.perf_counter() - t0
        futures = {}
        waiting = deque()  # arrived, not yet in a slot (per-size FIFO order)
        nxt = 0
        total = len(reqs)
        base = len(self.results)
        st = self.stats
        clock = time.perf_counter
        while len(self.results) - base < total:
            st["loop_passes"] += 1
            t = now()
            while nxt < total and (not realtime or reqs[nxt].arrival <= t):
                r = reqs[nxt]
                futures[r.rid] = pool.submit(prepare, r) if pool is not None else None
                waiting.append(r)
                nxt += 1
            still = deque()
            ta = clock()
            for r in waiting:
                f = futures[r.rid]
                g = self.groups[r.mesh]
                if not g.has_room() or (f is not None and not f.done()):
                    if g.has_room():
                        st["prep_waits"] += 1
                    still.append(r)
                    continue
                prep = f.result() if f is not None else prepare(r)
                del futures[r.rid]
                g.admit(r, prep, now())
                if r.want_grad:
                    self._grad.submit(r, prep)
            waiting = still
            st["admit_s"] += clock() - ta
            ran = False
            for g in self.groups.values():
                if g.n_active():
                    t1 = clock()
                    done = g.tick()
                    t2 = clock()
                    st["tick_s"] += t2 - t1
                    for b in done:
                        self._finalize(g, b)
                    st["finalize_s"] += clock() - t2
                    ran = True
            tc = clock()
            self._poll(now)
            st["poll_s"] += clock() - tc
            tc = clock()
            if not ran:
                if self._inflight:
                    self._inflight[0][0].synchronize()
                elif self._await_grad:
                    time.sleep(0.0005)
                elif nxt < total and realtime and not waiting:
                    time.sleep(max(0.0, min(0.002, reqs[nxt].arrival - now())))
                elif waiting:
                    time.sleep(0.0002)
            st["idle_s"] += clock() - tc
        return self.results


def run_plain(requests, realtime: bool = True, keep_density: bool | str = True, on_result=None):
    """The plain per-call path: one request at a time through the public API, FIFO
    (`keep_density` and `on_result` as for `Engine`)."""
    import jfli_b200 as jf

    reqs = sorted(requests, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    out = {}
    targets = {}
    solver = jf.EfficientDriftDoubleKick(interp_kernel=jf.NoInterp(painting=jf.PaintingOptions(target="density")))
    for r in reqs:
        if realtime and r.arrival > now():
            time.sleep(r.arrival - now())
        start = now()
        c = jf.Planck18(Omega_c=float(r.omega_c), sigma8=float(r.sigma8))
        noise = device_white_noise(r.seed, r.mesh)
        ic = jf.interpolate_initial_conditions(noise, (r.mesh,) * 3, (r.box,) * 3, cosmo=c)
        dx, p = jf.lpt(c, ic, ts=A_INIT, order=2)
        rho, run = jf.nbody(c, dx, p, t0=A_INIT, t1=1.0, dt0=(1.0 - A_INIT) / r.steps, solver=solver,
                            return_state=True)
        ps = rho.power(kedges=config_kedges(r.mesh, r.box))
        dens = rho.array if keep_density == "device" else (rho.array.cpu() if keep_density else None)
        pk = ps.array.cpu().numpy()
        res = ForwardResult(rid=r.rid, density=dens, k=ps.wavenumber.cpu().numpy(), pk=pk, steps=run.steps,
                            arrival=r.arrival, admitted=start)
        if r.want_grad:
            key = (r.mesh, r.box)
            if key not in targets:
                targets[key] = target_spectrum(*key)
            loss, gw, gom, gs8 = gradient_request(r, prepare(r), targets[key])
            res.loss, res.grad_noise, res.grad_omega_c, res.grad_sigma8 = float(loss), gw.cpu(), float(gom), float(gs8)
        res.done = now()
        if on_result is not None:
            on_result(res)
        out[r.rid] = res
    return out


def poisson_stream(n_requests: int, rate: float, seed: int = 0, grad_fraction: float = 0.25,
                   sizes=(64, 96, 128, 192)) -> list[ForwardRequest]:
    """The serving workload: Poisson arrivals, N ~ U{sizes}, L = 4 Mpc/h per cell,
    Omega_c ~ U[0.20, 0.35], sigma8 ~ U[0.70, 0.90], steps ~ U{10..40}, seed = request id."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests)) if rate > 0 else np.zeros(n_requests)
    out = []
    for i in range(n_requests):
        n = int(rng.choice(sizes))
        out.append(ForwardRequest(rid=i, mesh=n, box=4.0 * n, omega_c=float(rng.uniform(0.20, 0.35)),
                                  sigma8=float(rng.uniform(0.70, 0.90)), steps=int(rng.integers(10, 41)), seed=i,
                                  want_grad=bool(rng.random() < grad_fraction), arrival=float(t[i])))
    return out


def pk_max_rel(a: np.ndarray, b: np.ndarray) -> float:
    """Max per-bin relative difference of two P(k); bins with no modes (0 in both) count as equal."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_empty = (a == 0) & (b == 0)
    return float(np.max(np.where(both_empty, 0.0, np.abs(a / np.where(b == 0, 1.0, b) - 1))))


def summarize(results: dict, requests) -> dict:
    lat = np.array([results[r.rid].latency for r in requests]) * 1e3
    work = sum(r.mesh**3 * results[r.rid].steps for r in requests)
    start = min(r.arrival for r in requests)
    end = max(res.done for res in results.values())
    return {"requests": len(requests), "p50_ms": round(float(np.percentile(lat, 50)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2), "makespan_s": round(end - start, 3),
            "requests_per_s": round(len(requests) / (end - start), 1),
            "mpart_steps_per_s": round(work / (end - start) / 1e6, 1)}
