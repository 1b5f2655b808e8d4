"""Continuous-batching FFT serving loop over the B200 provider.

Requests of mixed lengths, batch counts, precisions, directions and normalizations arrive
over time. The server keeps plans and their tables resident on the device, admits waiting
requests while their buffers (and any new plan's scratch) fit an HBM budget, and launches
everything admitted so far without waiting for earlier work: requests whose length has a
size-specialised single-pass kernel are packed into one launch: power-of-two lengths up to
4096 (float) / 2048 (double) of every admitted request into one radix-family launch
(syclfft_b200_family_execute), other such lengths one grouped launch per length
(syclfft_b200_group_execute); the others run on resident plans made for any batch up to
512 (syclfft_b200_execute_ex), created ahead of admission by a worker
thread while the request waits. Families are spread over several CUDA
streams so independent work overlaps on the device. Latency is measured from a request's
arrival to the CUDA event that completes it. For comparison, the plain mode executes one
request at a time on the resident plans and waits for it, and the plan-per-request mode
does what a user of the plan API does for each request: create a plan for it, execute,
wait, destroy.
"""
from __future__ import annotations

import bisect
import ctypes
import math
import statistics
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _provider

ERR = 1024


@dataclass
class Request:
    rid: int
    lengths: tuple
    batch: int
    double: bool
    direction: int  # -1 forward, +1 backward
    normalization: int
    seed: int
    arrival: float  # seconds after the start of the run
    # filled while serving
    nbytes: int = 0
    t_done: float = 0.0
    in_ptr: int = 0   # device addresses of the request's input and output in the arena
    out_ptr: int = 0
    inp: object = None  # tensor views of them, made only when asked for (keep_results)
    out: object = None
    result: object = None

    @property
    def elements(self):
        return self.batch * math.prod(self.lengths)

    @property
    def flops(self):
        n = math.prod(self.lengths)
        return 5.0 * n * math.log2(n) * self.batch if n > 1 else 0.0


def _smooth7(n):
    for p in (2, 3, 5, 7):
        while n % p == 0:
            n //= p
    return n == 1


def _primes(lo, hi):
    sieve = np.ones(hi + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, int(hi ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    return [int(p) for p in np.nonzero(sieve)[0] if p >= lo]


def make_request_stream(count=20000, rate=50000.0, seed=5, max_batch=512, float_share=0.8):
    """The mixed request stream of the serving configuration: Poisson arrivals; lengths one
    third each from powers of two 2^6..2^20 (log-uniform), 7-smooth lengths and primes
    257..65537; batch log-uniform 1..512; 80% complex<float>; random direction and
    normalization; a per-request seed for the uniform[-1, 1) input."""
    rng = np.random.default_rng(seed)
    smooth = [n for n in range(64, 1 << 20) if _smooth7(n) and (n & (n - 1))]
    primes = _primes(257, 65537)
    t = 0.0
    reqs = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        fam = rng.integers(0, 3)
        if fam == 0:
            n = 1 << int(rng.integers(6, 21))
        elif fam == 1:
            n = int(smooth[int(np.exp(rng.uniform(0, np.log(len(smooth)))) - 1)])
        else:
            n = int(primes[int(rng.integers(0, len(primes)))])
        batch = int(np.clip(np.exp(rng.uniform(0, np.log(max_batch))), 1, max_batch))
        reqs.append(Request(i, (n,), batch, bool(rng.random() >= float_share), int(rng.choice([-1, 1])),
                            int(rng.integers(0, 4)), int(rng.integers(0, 2 ** 31)), t))
    return reqs


class Arena:
    """First-fit sub-allocator over one device buffer for the request buffers in flight: a
    request is admitted when its buffers fit, so admission tracks the real free space and no
    allocation or release during a run touches the CUDA allocator (whose retries after a
    failed allocation synchronize the device)."""

    ALIGN = 256

    def __init__(self, tensor):
        self.t = tensor
        self.size = tensor.numel()
        self.free = [(0, self.size)]  # (offset, bytes), sorted by offset, coalesced
        self.used = 0

    def alloc(self, nbytes):
        n = (nbytes + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        for i, (off, sz) in enumerate(self.free):
            if sz >= n:
                if sz == n:
                    del self.free[i]
                else:
                    self.free[i] = (off + n, sz - n)
                self.used += n
                return off
        return None

    def release(self, off, nbytes):
        n = (nbytes + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        self.used -= n
        i = bisect.bisect_left(self.free, (off, 0))
        self.free.insert(i, (off, n))
        # coalesce with the neighbours
        if i + 1 < len(self.free) and self.free[i][0] + self.free[i][1] == self.free[i + 1][0]:
            self.free[i] = (off, self.free[i][1] + self.free[i + 1][1])
            del self.free[i + 1]
        if i > 0 and self.free[i - 1][0] + self.free[i - 1][1] == self.free[i][0]:
            self.free[i - 1] = (self.free[i - 1][0], self.free[i - 1][1] + self.free[i][1])
            del self.free[i]

    def view(self, off, nbytes, dtype):
        return self.t[off: off + nbytes].view(dtype)


def _fill_items(reqs, lib=None):
    """FillItemV1 array of the requests' inputs (2 * elements reals each, at r.in_ptr)."""
    items = (_provider.FillItemV1 * len(reqs))()
    for i, r in enumerate(reqs):
        items[i].data = r.in_ptr
        items[i].count = 2 * r.elements
        items[i].seed = r.seed
        items[i].scalar = _provider.SCALAR_DOUBLE if r.double else _provider.SCALAR_FLOAT
    return items


def fill_inputs(reqs, stream_handle, lib=None):
    """Write every request's synthetic input (uniform[-1, 1) from its seed) at r.in_ptr, in one
    launch per 256 requests on the given raw stream."""
    if not reqs:
        return
    lib = lib or _provider.load()
    err = ctypes.create_string_buffer(ERR)
    if lib.syclfft_b200_fill_uniform(_fill_items(reqs), len(reqs), stream_handle, err, ERR):
        raise RuntimeError(err.value.decode())


def synthetic_input(r: Request, out=None):
    """The request's input: 2 * elements reals uniform in [-1, 1), value i a function of
    (r.seed, i) only (syclfft_b200_fill_uniform), viewed as complex; written into `out` when
    given, on the current stream."""
    import torch
    fdt = torch.float64 if r.double else torch.float32
    if out is None:
        out = torch.empty(2 * r.elements, device="cuda", dtype=fdt)
    q = Request(r.rid, r.lengths, r.batch, r.double, r.direction, r.normalization, r.seed, r.arrival)
    q.in_ptr = out.data_ptr()
    fill_inputs([q], torch.cuda.current_stream(out.device).cuda_stream)
    return torch.view_as_complex(out.view(-1, 2))


def _pow2_ceil(v):
    return 1 << max(0, (int(v) - 1).bit_length())


class Server:
    """`budget_bytes` bounds the request buffers in flight; `plan_budget_bytes` bounds the
    resident plans (least recently used plans are released once their last launch is done)."""

    def __init__(self, device=None, budget_bytes=120e9, streams=4, plan_budget_bytes=16e9, plan_workers=2):
        import torch
        from collections import OrderedDict
        self.torch = torch
        self.dev = torch.cuda.current_device() if device is None else device
        self.lib = _provider.load()
        self.api = _provider.provider(self.lib)
        self.budget = float(budget_bytes)
        self.plan_workers = int(plan_workers)  # threads creating plans ahead of admission
        self.plan_budget = float(plan_budget_bytes)
        self.streams = [torch.cuda.Stream(self.dev) for _ in range(streams)]
        # (lengths, double, batch class) -> [handle, bytes, last launch event]; both directions
        # and every normalization run on one plan (syclfft_b200_execute_ex)
        self.plans = OrderedDict()
        self.retired = []   # (handle, event): released when the event has completed
        self.groups = {}    # (n, double) -> handle
        self.families = {}  # double -> radix-family handle (power-of-two lengths of one launch)
        self.err = ctypes.create_string_buffer(ERR)
        self.plan_bytes = 0
        self.plans_created = 0
        self.evictions = 0
        self.max_waiting = 0
        self.pending = {}   # plan key -> future of a plan being created ahead of use
        self.pool = None
        self.arena = None   # request buffers of a run (Arena)

    # ---------------------------------------------------------------- resident state
    MAX_BATCH = 512

    def _create(self, lengths, double):
        """Create a resident plan (tables only; any batch up to MAX_BATCH). Thread-safe: called
        from the plan-prefetch worker too (ctypes releases the GIL during creation)."""
        err = ctypes.create_string_buffer(ERR)
        cfg = _provider.make_config(list(lengths), self.MAX_BATCH, -1, double, False, 0, False, self.dev)
        # scratch comes from the executing stream's arena; creation does not block on the device
        handle = self.lib.syclfft_b200_create_ex(ctypes.byref(cfg), _provider.CREATE_STREAM_SCRATCH, err, ERR)
        if not handle:
            raise RuntimeError(err.value.decode())
        return handle

    def _prefetch(self, r: Request):
        key = (r.lengths, r.double)
        if key in self.plans or key in self.pending or self.pool is None or self.groupable(r) or self.family_member(r):
            return
        self.pending[key] = self.pool.submit(self._create, r.lengths, r.double)

    def _plan(self, r: Request):
        key = (r.lengths, r.double)
        h = self.plans.get(key)
        if h is not None:
            self.plans.move_to_end(key)
            return h
        fut = self.pending.pop(key, None)
        handle = fut.result() if fut is not None else self._create(r.lengths, r.double)
        nbytes = int(self.lib.syclfft_b200_plan_device_bytes(handle))  # the plan's tables
        h = [handle, nbytes, None]
        self.plans[key] = h
        self.plan_bytes += nbytes
        self.plans_created += 1
        return h

    def _evict(self):
        """Release least recently used plans over the plan budget once their last launch is
        done. Called after a round's launches are enqueued, so no plan of the round is released
        before its execute is issued (the release itself is ordered after it on the device)."""
        while self.plan_bytes > self.plan_budget and len(self.plans) > 1:
            _, (oh, ob, oev) = self.plans.popitem(last=False)
            self.plan_bytes -= ob
            self.retired.append((oh, oev))
            self.evictions += 1
        self._reap()

    def _reap(self, wait=False):
        keep = []
        for handle, ev in self.retired:
            if ev is None or wait or ev.query():
                if ev is not None and wait:
                    ev.synchronize()
                self.api.destroy(handle)
            else:
                keep.append((handle, ev))
        self.retired = keep

    def _group(self, n, double):
        key = (n, double)
        g = self.groups.get(key)
        if g is None:
            g = self.lib.syclfft_b200_group_create(2 if double else 1, n, self.dev, self.err, ERR)
            if not g:
                raise RuntimeError(self.err.value.decode())
            self.groups[key] = g
        return g

    def _family(self, double):
        f = self.families.get(double)
        if f is None:
            f = self.lib.syclfft_b200_family_create(2 if double else 1, self.dev, self.err, ERR)
            if not f:
                raise RuntimeError(self.err.value.decode())
            self.families[double] = f
        return f

    def family_member(self, r: Request):
        """Lengths served by the radix-family launch: several lengths in one kernel."""
        return len(r.lengths) == 1 and bool(self.lib.syclfft_b200_family_supports(2 if r.double else 1,
                                                                                  r.lengths[0]))

    def groupable(self, r: Request):
        return len(r.lengths) == 1 and bool(self.lib.syclfft_b200_group_supports(2 if r.double else 1, r.lengths[0]))

    def close(self):
        for fut in self.pending.values():
            self.api.destroy(fut.result())
        self.pending.clear()
        self.torch.cuda.synchronize(self.dev)
        self._reap(wait=True)
        for st in self.streams:  # the plans' scratch arenas on this server's streams
            self.lib.syclfft_b200_release_stream_scratch(st.cuda_stream, self.dev)
        for handle, _, _ in self.plans.values():
            self.api.destroy(handle)
        for g in self.groups.values():
            self.lib.syclfft_b200_group_destroy(g)
        for f in self.families.values():
            self.lib.syclfft_b200_family_destroy(f)
        self.plans.clear()
        self.groups.clear()
        self.families.clear()
        self.arena = None
        # hand the request buffers cached by torch back to the device for other pools
        self.torch.cuda.empty_cache()

    # ---------------------------------------------------------------- data
    def _views(self, r: Request):
        """Tensor views of a request's input and output in the arena (made on demand)."""
        torch = self.torch
        fdt = torch.float64 if r.double else torch.float32
        buf = self.arena.view(r.buf_off, r.nbytes, fdt)
        r.inp = torch.view_as_complex(buf[: 2 * r.elements].view(-1, 2))
        r.out = torch.view_as_complex(buf[2 * r.elements:].view(-1, 2))

    def _reserve(self, r: Request):
        off = self.arena.alloc(r.nbytes)
        if off is not None:
            r.buf_off = off
            r.in_ptr = self.arena_base + off
            r.out_ptr = r.in_ptr + r.nbytes // 2
        return off is not None

    def _release(self, r: Request):
        self.arena.release(r.buf_off, r.nbytes)
        r.inp = r.out = None

    def _fill(self, reqs, stream):
        fill_inputs(reqs, stream.cuda_stream, self.lib)

    def _execute_plans(self, reqs, stream):
        """The requests on their resident plans, one native call (syclfft_b200_execute_many)."""
        items = (_provider.ExecItemV1 * len(reqs))()
        used = []
        for i, r in enumerate(reqs):
            h = self._plan(r)
            used.append(h)
            items[i].plan = h[0]
            items[i].in_ = r.in_ptr
            items[i].out = r.out_ptr
            items[i].batch = r.batch
            items[i].direction = r.direction
            items[i].normalization = r.normalization
        if self.lib.syclfft_b200_execute_many(items, len(reqs), stream.cuda_stream, self.err, ERR):
            raise RuntimeError(self.err.value.decode())
        self._evict()
        return used

    def _execute_family(self, double, reqs, stream):
        f = self._family(double)
        items = (_provider.FamilyItemV1 * len(reqs))()
        for i, r in enumerate(reqs):
            items[i].in_ = r.in_ptr
            items[i].out = r.out_ptr
            items[i].n = r.lengths[0]
            items[i].batch = r.batch
            items[i].direction = r.direction
            items[i].normalization = r.normalization
        rc = self.lib.syclfft_b200_family_execute(f, items, len(reqs), stream.cuda_stream, self.err, ERR)
        if rc:
            raise RuntimeError(self.err.value.decode())

    def _execute_group(self, key, reqs, stream):
        n, double = key
        g = self._group(n, double)
        items = (_provider.GroupItemV1 * len(reqs))()
        for i, r in enumerate(reqs):
            items[i].in_ = r.in_ptr
            items[i].out = r.out_ptr
            items[i].batch = r.batch
            items[i].direction = r.direction
            items[i].normalization = r.normalization
        rc = self.lib.syclfft_b200_group_execute(g, items, len(reqs), stream.cuda_stream, self.err, ERR)
        if rc:
            raise RuntimeError(self.err.value.decode())

    # ---------------------------------------------------------------- loops
    def _keep(self, r: Request, keep_results):
        """What a run keeps of a finished request's output before its buffer is reused: all of
        it on the host (keep_results True) or what a callable returns for it."""
        if not keep_results:
            return
        self._views(r)
        if callable(keep_results):
            r.result = keep_results(r)
        else:
            r.result = r.out.cpu()

    def run(self, requests, mode="served", keep_results=False):
        """Serve `requests` (sorted by arrival); returns statistics. mode 'served' (continuous
        batching), 'plain' (one request at a time on resident plans) or 'plan_per_request'
        (one request at a time, each with its own plan created and destroyed around it).
        keep_results: False, True (every output copied to the host into r.result) or a
        callable f(request) -> r.result, called once the output is complete."""
        torch = self.torch
        self.evictions = 0
        self.max_waiting = 0
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            r.nbytes = 2 * r.elements * (16 if r.double else 8)
        start = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(self.dev)
        torch.cuda.empty_cache()
        # the admission budget as one arena for the request buffers, leaving room for resident
        # plans and the streams' scratch arenas (CUDA memory pool)
        free, _ = torch.cuda.mem_get_info(self.dev)
        size = int(min(self.budget, free - self.plan_budget - 8e9))
        if size < max(r.nbytes for r in reqs):
            raise RuntimeError("admission budget smaller than the largest request")
        self.arena = Arena(torch.empty(size, dtype=torch.uint8, device=f"cuda:{self.dev}"))
        self.arena_base = self.arena.t.data_ptr()
        torch.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        start.record(self.streams[0])
        done_events = []
        if mode == "plan_per_request":
            # The reference's usage: a plan for each request's exact shape, batch, direction
            # and normalization, one execute, wait, destroy.
            s = self.streams[0]
            for r in reqs:
                while time.perf_counter() - t0 < r.arrival:
                    pass
                self._reserve(r)
                self._fill([r], s)
                cfg = _provider.make_config(list(r.lengths), r.batch, r.direction, r.double, False, r.normalization,
                                            False, self.dev)
                h = self.api.create(ctypes.byref(cfg), self.err, ERR)
                if not h:
                    raise RuntimeError(self.err.value.decode())
                self.plans_created += 1
                rc = self.api.execute(h, r.in_ptr, r.out_ptr, s.cuda_stream, self.err, ERR)
                if rc:
                    raise RuntimeError(self.err.value.decode())
                with torch.cuda.stream(s):
                    ev = torch.cuda.Event(enable_timing=True)
                    ev.record(s)
                ev.synchronize()
                self.api.destroy(h)
                r.t_done = start.elapsed_time(ev) / 1e3
                self._keep(r, keep_results)
                self._release(r)
        elif mode == "plain":
            s = self.streams[0]
            for r in reqs:
                while time.perf_counter() - t0 < r.arrival:
                    pass
                self._reserve(r)
                self._fill([r], s)
                h = self._execute_plans([r], s)[0]
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(s)
                h[2] = ev
                ev.synchronize()
                r.t_done = start.elapsed_time(ev) / 1e3
                self._keep(r, keep_results)
                self._release(r)
        else:
            self._serve(reqs, t0, start, keep_results)
        torch.cuda.synchronize(self.dev)
        lat = [r.t_done - r.arrival for r in reqs]
        makespan = max(r.t_done for r in reqs) - min(r.arrival for r in reqs)
        total_flops = sum(r.flops for r in reqs)
        total_bytes = sum(r.nbytes for r in reqs)
        lat_sorted = sorted(lat)
        return {
            "mode": mode, "requests": len(reqs), "makespan_s": makespan,
            "throughput_gflops": total_flops / makespan / 1e9, "throughput_gbs": total_bytes / makespan / 1e9,
            "requests_per_s": len(reqs) / makespan,
            "p50_ms": 1e3 * lat_sorted[len(lat) // 2], "p99_ms": 1e3 * lat_sorted[min(len(lat) - 1, int(0.99 * len(lat)))],
            "mean_ms": 1e3 * statistics.mean(lat), "plans_resident": len(self.plans),
            "plans_created": self.plans_created, "groups": len(self.groups), "families": len(self.families),
            "plan_bytes": self.plan_bytes, "plan_evictions": self.evictions, "max_waiting": self.max_waiting,
        }

    def _serve(self, reqs, t0, start, keep_results):
        from concurrent.futures import ThreadPoolExecutor
        self.pool = ThreadPoolExecutor(max_workers=self.plan_workers)
        try:
            self._serve_loop(reqs, t0, start, keep_results)
        finally:
            self.pool.shutdown(wait=True)
            self.pool = None

    ADMIT_WINDOW = 64      # requests behind a head that does not fit that may be admitted first
    HEAD_PATIENCE = 0.05   # seconds a head may be passed over before everything waits for it

    def _serve_loop(self, reqs, t0, start, keep_results):
        torch = self.torch
        nxt = 0
        head_blocked = None  # when the current head first failed to fit
        waiting = deque()
        S = len(self.streams)
        in_flight = [deque() for _ in range(S)]  # per stream, in launch order: (event, [requests])
        completed = 0
        while completed < len(reqs):
            now = time.perf_counter() - t0
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                waiting.append(reqs[nxt])
                self._prefetch(reqs[nxt])  # start its plan while it waits for admission
                nxt += 1
            self.max_waiting = max(self.max_waiting, len(waiting))
            # admission by HBM budget: FIFO while the request's buffers fit in the arena; when the
            # head does not fit, up to ADMIT_WINDOW requests behind it that do fit go ahead (the
            # GPU would otherwise idle behind one large request), unless the head has already
            # been passed over for HEAD_PATIENCE seconds, which keeps it from starving
            bins = {}
            admitted = []
            i = skipped = 0
            while i < len(waiting) and skipped <= self.ADMIT_WINDOW:
                r = waiting[i]
                if self._reserve(r):
                    admitted.append(r)
                    del waiting[i]
                    if i == 0:
                        head_blocked = None
                    continue
                if i == 0:
                    if head_blocked is None:
                        head_blocked = now
                    elif now - head_blocked > self.HEAD_PATIENCE:
                        break
                skipped += 1
                i += 1
            for r in admitted:
                if self.family_member(r):
                    key = ("f", r.double)
                elif self.groupable(r):
                    key = ("g", r.lengths[0], r.double)
                else:
                    key = ("p", r.lengths, r.double)
                bins.setdefault(key, []).append(r)
            # launch everything admitted: one grouped launch per length family
            for key, rs in bins.items():
                si = hash(key) % S
                s = self.streams[si]
                used_plans = []
                self._fill(rs, s)
                if key[0] == "f":
                    self._execute_family(key[1], rs, s)
                elif key[0] == "g":
                    self._execute_group((key[1], key[2]), rs, s)
                else:
                    used_plans = self._execute_plans(rs, s)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(s)
                for h in used_plans:
                    h[2] = ev
                in_flight[si].append((ev, rs))
            # completions: work on one stream completes in launch order, so only each
            # stream's oldest launch needs polling
            progressed = False
            for q in in_flight:
                while q and q[0][0].query():
                    ev, rs = q.popleft()
                    t = start.elapsed_time(ev) / 1e3
                    for r in rs:
                        r.t_done = t
                        self._keep(r, keep_results)
                        self._release(r)
                    completed += len(rs)
                    progressed = True
            if progressed and self.retired:
                self._reap()
            if not progressed and not bins:
                busy = [q for q in in_flight if q]
                if busy and (waiting or nxt >= len(reqs)):
                    # blocked on memory or draining: wait for the oldest launch of a busy stream
                    busy[0][0][0].synchronize()
                elif nxt < len(reqs):
                    # idle until the next arrival (short sleeps keep arrival times honest)
                    gap = reqs[nxt].arrival - (time.perf_counter() - t0)
                    if gap > 2e-4:
                        time.sleep(min(gap, 1e-3))
