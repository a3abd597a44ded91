"""Served form: a request loop with continuous batching on one GPU.

Jobs (``JobSpec``) arrive at any time.  The server

* admits a job when its HBM footprint (``engine.estimate_device_bytes``) fits
  the remaining budget and an execution slot is free -- jobs that arrive while
  others are on the GPU are admitted as soon as slots and memory free up;
* keeps every admitted job's sky, beams, Z panel and partial visibilities
  resident on the device, and gives it its own CUDA stream;
* advances the active jobs in turns, so their kernels overlap on the device,
  with at most ``turns_ahead`` turns enqueued ahead of the GPU (so a job
  admitted now starts behind a bounded backlog).  A turn takes the jobs with
  the least estimated work left first, until their next groups add up to
  ``turn_terms`` terms (a job passed over ``max_skipped`` turns in a row is
  taken regardless; ``turn_terms=None`` is plain round robin): each chosen
  job's next group of frequencies gets its tau/Z on
  the job's stream, and the Hermitian products of all those groups run in one
  launch (``mvb_herk_batch``, up to 32 panels) on a shared stream, ordered
  against the jobs' streams by events; each job then reduces its own group
  (jobs whose product cannot be batched -- pair lists on per-pair sums, beamfits
  beams -- advance a time step per turn on their own stream);
* optionally (``small_job_terms``) treats jobs below a size as a priority
  class: they are admitted ahead of larger pending jobs and run on
  high-priority streams, whose thread blocks the GPU dispatches first as SMs
  free up, so a short job does not wait behind a long one; larger jobs keep
  their arrival order;
* defers a job whose buffers the allocator cannot place (fragmentation) until
  another job retires, and fails it alone only if nothing else holds memory;
* hands each finished job to a copier thread, which waits for the job's last
  kernel on its own stream, copies the visibilities and the status word to the
  host (touching the result's pages first), and counts the job's terms, so the
  scheduling loop never waits on a copy or a host allocation; the job's latency
  runs from submission to its result on the host, after which its device
  memory is freed.

Each job's arithmetic is exactly the single-job path (same kernels, same
deterministic reduction order), so a result is bit-identical alone and in a
mix.  ``latency_summary`` reports p50 / p99 and the throughput.
"""

from __future__ import annotations

import os
import queue
import threading
import time
from collections import deque
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .engine import JobSpec, VisEngine, estimate_device_bytes

# The jobs' streams map onto the device's hardware work queues, 8 by default;
# with more active jobs than queues, kernels of unrelated jobs serialise behind
# each other.  32 queues measured p50 1.27 s against 2.18 s on the 2,000-job
# config-5 stream at 8 active jobs.  Only effective before the process's first
# CUDA call (set it in the environment otherwise).
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")


@dataclass
class _Job:
    jid: int
    spec: JobSpec
    t_submit: float
    engine: VisEngine | None = None
    stream: torch.cuda.Stream | None = None
    next_t: int = 0
    done_event: torch.cuda.Event | None = None
    host: np.ndarray | None = None
    status_word: int = 0
    footprint: int = 0
    small: bool = False
    #: next (time, source chunk, first frequency) of a batched job, and its beam buffer
    cursor: tuple = (0, 0, 0)
    beam: torch.Tensor | None = None
    t_admit: float = 0.0
    t_done: float = 0.0
    terms: float = 0.0
    error: str | None = None
    #: estimated terms of one frequency group, and turns passed over in a row
    group_terms: float = 0.0
    skipped: int = 0


@dataclass
class JobResult:
    jid: int
    vis: np.ndarray | None
    latency_s: float
    queue_s: float
    terms: float
    error: str | None = None


class VisServer:
    """Continuous-batching visibility server on one device."""

    def __init__(self, device=None, hbm_budget: int | None = None, max_active: int = 32, steps_per_turn: int = 1,
                 reserve_fraction: float = 0.0, keep_results: bool = True, small_job_terms: float | None = 2e11,
                 batch_products: bool = True, turns_ahead: int | None = 2, turn_terms: float | None = 2e11,
                 max_skipped: int = 8):
        self.device = _lib.require_cuda(device)
        free = torch.cuda.mem_get_info(self.device)[0]
        # 0.75 of the free memory: at 0.85 the caching allocator's fragmentation
        # made admissions run out of memory several times more often
        self.budget = int(hbm_budget if hbm_budget is not None else 0.75 * free)
        # every admitted job's buffers are allocated on this one stream, so the
        # caching allocator hands a finished job's blocks to the next job (blocks
        # are cached per allocating stream; a fresh stream per job would strand
        # them, until an out-of-memory retry frees the whole cache with a device
        # synchronisation).  A job's buffers are freed only after its last
        # kernel has completed, so any stream may reuse them.
        self._alloc_stream = torch.cuda.Stream(device=self.device)
        # optionally, a block of the budget taken once and handed back to the
        # cache of that stream, for jobs to be carved from (fewer cudaMalloc
        # calls, at the risk of fragmenting one segment that can then never be
        # released: off by default)
        if reserve_fraction > 0:
            with torch.cuda.stream(self._alloc_stream):
                reserve = torch.empty(int(self.budget * min(reserve_fraction, 1.0)), dtype=torch.uint8,
                                      device=self.device)
                del reserve
        self.max_active = max_active
        self.steps_per_turn = steps_per_turn
        #: turns enqueued on the device and not yet complete before the server
        #: waits to enqueue another (None: no bound).  Without a bound the host
        #: runs ahead of the GPU and a newly admitted job's first kernels queue
        #: behind every turn already enqueued for the others.
        self.turns_ahead = turns_ahead
        self._turns: deque[list] = deque()
        #: None: every active job advances each turn (round robin).  Otherwise a
        #: turn takes the batched jobs with the least estimated work left first,
        #: until their groups add up to this many terms; a job passed over
        #: max_skipped turns in a row is taken regardless.
        self.turn_terms = turn_terms
        self.max_skipped = max_skipped
        #: admissions that ran out of device memory (retried later), and the
        #: memory in use when the last one did
        self.oom_retries = 0
        self._oom_wait: int | None = None
        self._turn: list = []  # events that complete the turn being enqueued
        #: False: results keep the latency and term count only (a long benchmark stream)
        self.keep_results = keep_results
        #: kernel launches made for the admitted jobs (shared product launches counted once)
        self.launches = 0
        #: jobs of at most this many (estimated) terms form the priority class
        self.small_job_terms = small_job_terms
        self._small: deque[_Job] = deque()
        #: run the products of the active jobs' current frequency groups in shared launches
        self.batch_products = batch_products
        self._batch_streams = {False: torch.cuda.Stream(device=self.device),
                               True: torch.cuda.Stream(device=self.device, priority=-1)}
        #: product launches (mvb_herk_batch) and the panel groups they carried
        self.batch_launches = 0
        self.batched_groups = 0
        self._pending: deque[_Job] = deque()
        self._active: list[_Job] = []
        self._finishing: list[_Job] = []
        self._results: dict[int, JobResult] = {}
        self._lock = threading.Lock()
        self._next_id = 0
        self.in_use = 0
        self.peak_in_use = 0
        self.max_concurrent = 0
        self._to_copy: queue.Queue = queue.Queue()
        self._copied: queue.Queue = queue.Queue()
        self._copier = threading.Thread(target=self._copy_loop, name="mvb-serve-d2h", daemon=True)
        self._copier.start()

    def close(self):
        """Stop the copier thread (the server serves no more jobs after this)."""
        if self._copier.is_alive():
            self._to_copy.put(None)
            self._copier.join()

    def _copy_loop(self):
        torch.cuda.set_device(self.device)
        cs = torch.cuda.Stream(device=self.device)
        status = torch.empty(1, dtype=torch.int32, pin_memory=True)
        while (job := self._to_copy.get()) is not None:
            try:
                eng = job.engine
                host = np.empty(tuple(eng.vis.shape), dtype=np.complex64 if eng.vis.dtype == torch.complex64
                                else np.complex128)
                host.reshape(-1)[:: 4096 // host.itemsize] = 0  # first-touch the pages before the copy
                with torch.cuda.stream(cs):
                    cs.wait_event(job.done_event)
                    torch.from_numpy(host).copy_(eng.vis)  # pageable destination: returns when done
                    status.copy_(eng.status)
                    cs.synchronize()
                job.status_word = int(status[0])
                job.host = host
                job.t_done = time.perf_counter()
                job.terms = float(eng.nant ** 2 * len(eng.freqs)) * self._n_above_total(job)
            except Exception as exc:  # recorded per job; the server keeps running
                job.error = f"copy failed: {exc}"
                job.t_done = time.perf_counter()
            self._copied.put(job)

    # ------------------------------------------------------------------ API
    def submit(self, spec: JobSpec, t_submit: float | None = None) -> int:
        fp = estimate_device_bytes(spec)
        if fp > self.budget:
            raise ValueError(f"job needs {fp / 1e9:.2f} GB of HBM, more than the server budget {self.budget / 1e9:.2f} GB")
        with self._lock:
            jid = self._next_id
            self._next_id += 1
            job = _Job(jid=jid, spec=spec, t_submit=time.perf_counter() if t_submit is None else t_submit, footprint=fp)
            small = self.small_job_terms is not None and estimate_terms(spec) <= self.small_job_terms
            (self._small if small else self._pending).append(job)
            job.small = small
        return jid

    def result(self, jid: int) -> JobResult | None:
        return self._results.get(jid)

    @property
    def results(self) -> dict[int, JobResult]:
        return self._results

    def idle(self) -> bool:
        with self._lock:
            return not self._pending and not self._small and not self._active and not self._finishing

    # ------------------------------------------------------------ scheduling
    def _admit(self):
        with self._lock:
            while len(self._active) < self.max_active:
                # the priority class first, each class in arrival order
                q = self._small if self._small else self._pending
                if not q:
                    break
                job = q[0]
                if self.in_use + job.footprint > self.budget:
                    break
                if self._oom_wait is not None and self.in_use >= self._oom_wait:
                    break  # the last admission ran out of device memory: wait for jobs to retire
                self._oom_wait = None
                if not self._allocate(job):
                    if self._active or self._finishing:
                        # the budget has room but the allocator could not place the
                        # job's buffers: keep it at the head of its queue until a job
                        # retires
                        self._oom_wait = self.in_use
                        break
                    # nothing else holds device memory: the job cannot run here
                    q.popleft()
                    now = time.perf_counter()
                    self._results[job.jid] = JobResult(jid=job.jid, vis=None, latency_s=now - job.t_submit,
                                                       queue_s=now - job.t_submit, terms=0.0,
                                                       error="out of device memory at admission")
                    continue
                q.popleft()
                self.in_use += job.footprint
                self.peak_in_use = max(self.peak_in_use, self.in_use)
                job.t_admit = time.perf_counter()
                job.stream = torch.cuda.Stream(device=self.device, priority=-1 if job.small else 0)
                job.stream.wait_stream(self._alloc_stream)  # the buffers' zero fills
                with torch.cuda.stream(job.stream):
                    job.engine.upload()
                    job.engine.status.zero_()
                eng = job.engine
                ngroups = len(eng.lsts) * eng.nchunks * -(-len(eng.freqs) // max(eng.fgroup, 1))
                job.group_terms = estimate_terms(job.spec) / max(ngroups, 1)
                self.launches += eng.launches_per_run()
                if self.batch_products and eng.batchable:
                    # its product launches are shared ones, counted as they are made
                    self.launches -= len(eng.lsts) * eng.nchunks * -(-len(eng.freqs) // max(eng.fgroup, 1))
                self._active.append(job)
        self.max_concurrent = max(self.max_concurrent, len(self._active))

    def _allocate(self, job: _Job) -> bool:
        """The job's engine and device buffers, on the allocation stream; False
        (nothing kept) when the device cannot hold them (torch's allocator has
        already released its unused cached blocks and retried before it raises)."""
        try:
            with torch.cuda.stream(self._alloc_stream):
                job.engine = VisEngine(job.spec, device=self.device)
                job.engine.allocate()
            return True
        except torch.OutOfMemoryError:
            job.engine = None
            self.oom_retries += 1
            return False

    def _throttled(self) -> bool:
        """True while turns_ahead turns are enqueued and not yet complete."""
        if self.turns_ahead is None:
            return False
        while self._turns and all(e.query() for e in self._turns[0]):
            self._turns.popleft()
        return len(self._turns) >= self.turns_ahead

    def _advance(self):
        if self._throttled():
            return
        self._turn = []
        still = []
        batch = []
        chosen = self._choose_batched()
        for job in self._active:
            eng = job.engine
            if self.batch_products and eng.batchable:
                if chosen is not None and job.jid not in chosen:
                    job.skipped += 1
                    still.append(job)
                    continue
                job.skipped = 0
                # this turn: the job's next frequency group up to its product
                t, c, f0 = job.cursor
                if t >= len(eng.lsts):  # no time steps at all
                    self._finish(job)
                    continue
                with torch.cuda.stream(job.stream):
                    if f0 == 0:
                        job.beam = eng.chunk_prologue(t, c, stream=job.stream)
                    g = eng.tau_z_group(t, f0, job.beam, stream=job.stream)
                    ready = torch.cuda.Event()
                    ready.record(job.stream)
                batch.append((job, g, ready))
                continue
            nt = len(eng.lsts)
            with torch.cuda.stream(job.stream):
                for _ in range(self.steps_per_turn):
                    if job.next_t >= nt:
                        break
                    eng.enqueue_time(job.next_t, stream=job.stream)
                    job.next_t += 1
                step_done = torch.cuda.Event()
                step_done.record(job.stream)
                self._turn.append(step_done)
                if job.next_t >= nt:
                    self._finish(job)
                    continue
            still.append(job)
        self._active = still + (self._launch_batches(batch) if batch else [])
        if self._turn:
            self._turns.append(self._turn)

    def _remaining_terms(self, job: _Job) -> float:
        eng = job.engine
        t, c, f0 = job.cursor
        per_t = eng.nchunks * -(-len(eng.freqs) // max(eng.fgroup, 1))
        done = t * per_t + c * -(-len(eng.freqs) // max(eng.fgroup, 1)) + f0 // max(eng.fgroup, 1)
        return (len(eng.lsts) * per_t - done) * job.group_terms

    def _choose_batched(self) -> set | None:
        """The batched jobs that advance this turn (None: all of them)."""
        if self.turn_terms is None or not self.batch_products:
            return None
        jobs = [j for j in self._active if j.engine.batchable]
        if not jobs:
            return None
        chosen, total = set(), 0.0
        for j in sorted(jobs, key=lambda j: (j.skipped < self.max_skipped, self._remaining_terms(j))):
            if chosen and total + j.group_terms > self.turn_terms and j.skipped < self.max_skipped:
                continue
            chosen.add(j.jid)
            total += j.group_terms
        return chosen

    def _finish(self, job: _Job):
        """The job's last kernel is enqueued: hand it to the copier."""
        job.done_event = torch.cuda.Event()
        job.done_event.record(job.stream)
        self._finishing.append(job)
        self._to_copy.put(job)

    def _launch_batches(self, batch: list) -> list:
        """The products of this turn's groups, in launches of at most 32 panels
        per (split mode, drain interval, priority class); then each job's
        reduction on its own stream.  Returns the jobs still active."""
        packs: dict = {}
        for item in batch:
            eng = item[0].engine
            packs.setdefault((eng.matprod.mode, eng.matprod.drain_ksteps, item[0].small), []).append(item)
        still = []
        for (mode, kd, small), items in packs.items():
            while items:
                take, n = [], 0
                while items and n + items[0][1] <= _lib.MAX_BATCH_PANELS:
                    take.append(items.pop(0))
                    n += take[-1][1]
                bs = self._batch_streams[small]
                groups = (_lib.HerkGroup * len(take))()
                for i, (job, g, ready) in enumerate(take):
                    bs.wait_event(ready)
                    eng = job.engine
                    groups[i] = eng.matprod.batch_group(eng.panels[:g], eng.k_chunk)
                _lib.check(_lib.lib.mvb_herk_batch(_lib.c_void_p(_lib.ctypes.addressof(groups)), len(take), mode, kd,
                                                   _lib.stream_handle(bs)))
                done = torch.cuda.Event()
                done.record(bs)
                self._turn.append(done)
                self.batch_launches += 1
                self.launches += 1
                self.batched_groups += len(take)
                for job, g, _ in take:
                    if self._reduce_and_step(job, g, done):
                        still.append(job)
        return still

    def _reduce_and_step(self, job: _Job, g: int, done: torch.cuda.Event) -> bool:
        """The job's reduction of its batched group, then its cursor moves on;
        False once the job has enqueued its last kernel."""
        eng = job.engine
        t, c, f0 = job.cursor
        job.stream.wait_event(done)
        with torch.cuda.stream(job.stream):
            eng.matprod.reduce_grouped(eng.panels[:g], eng.vis[f0:f0 + g, t], accumulate=c > 0, stream=job.stream,
                                       k_chunk=eng.k_chunk)
        f0 += g
        if f0 >= len(eng.freqs):
            f0, c = 0, c + 1
            if c >= eng.nchunks:
                c, t = 0, t + 1
        job.cursor = (t, c, f0)
        if t >= len(eng.lsts):
            self._finish(job)
            return False
        return True

    def _retire(self):
        while True:
            try:
                job = self._copied.get_nowait()
            except queue.Empty:
                break
            err = job.error
            if err is None and job.status_word:
                try:
                    _lib.check_status_word(torch.tensor([job.status_word], dtype=torch.int32), f"job {job.jid}")
                except Exception as exc:
                    err = str(exc)
            vis = job.host
            if vis is not None and not job.spec.polarized:
                vis = vis[..., 0, 0]
            if not self.keep_results:
                vis = None
            self._results[job.jid] = JobResult(jid=job.jid, vis=None if err else vis, latency_s=job.t_done - job.t_submit,
                                               queue_s=job.t_admit - job.t_submit, terms=job.terms, error=err)
            job.spec = None
            with self._lock:
                self.in_use -= job.footprint
            self._finishing.remove(job)
            job.engine = None
            job.stream = None
            job.host = None

    @staticmethod
    def _n_above_total(job: _Job) -> float:
        """Sum over times of the above-horizon counts (host FP64 rotation, same op order)."""
        eng = job.engine
        eci = eng.eci_host
        tot = 0
        for R in eng.rot:
            z = (R[2, 0] * eci[0] + R[2, 1] * eci[1]) + R[2, 2] * eci[2]
            tot += int((z > 0).sum())
        return float(tot)

    def poll(self):
        """One scheduling turn: admit, advance every active job by a time step, retire."""
        self._admit()
        self._advance()
        self._retire()

    def run_until_idle(self, timeout_s: float = 3600.0):
        t0 = time.perf_counter()
        while not self.idle():
            self.poll()
            if (not self._active and self._finishing) or self._throttled():
                time.sleep(0.0005)
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError("server did not drain in time")

    def serve_stream(self, arrivals, timeout_s: float = 3600.0) -> list[int]:
        """Submit jobs at their arrival offsets (seconds from now) while serving.

        ``arrivals``: (offset_s, JobSpec) pairs -- a list (sorted here) or any
        iterable in non-decreasing offset order, e.g. a generator that builds
        each job only when its turn comes, so a long stream never holds all its
        skies in host memory at once."""
        t0 = time.perf_counter()
        ids = []
        it = iter(sorted(arrivals, key=lambda a: a[0]) if isinstance(arrivals, list) else arrivals)
        nxt = next(it, None)
        while nxt is not None or not self.idle():
            now = time.perf_counter() - t0
            while nxt is not None and nxt[0] <= now:
                ids.append(self.submit(nxt[1], t_submit=t0 + nxt[0]))
                nxt = next(it, None)
            if self.idle() and nxt is not None:
                time.sleep(min(0.001, max(0.0, nxt[0] - now)))
                continue
            self.poll()
            if (not self._active and self._finishing and not self._pending) or self._throttled():
                time.sleep(0.0002)  # copies or enqueued turns in flight: leave the interpreter to the copier
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError("serve_stream did not finish in time")
        return ids


def estimate_terms(spec: JobSpec) -> float:
    """Antenna-pair x source terms of a job, with half the sky above the horizon
    (for scheduling; the reported counts are exact)."""
    npairs = len(spec.antpos) ** 2 if spec.antpairs is None else len(spec.antpairs)
    return float(npairs) * 0.5 * np.asarray(spec.eci).shape[1] * len(spec.freqs) * len(spec.lsts)


def latency_summary(results: dict[int, JobResult]) -> dict:
    ok = [r for r in results.values() if r.error is None]
    if not ok:
        return {"jobs": 0}
    lat = np.array([r.latency_s for r in ok])
    q = np.array([r.queue_s for r in ok])
    return {
        "jobs": len(ok),
        "errors": len(results) - len(ok),
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
        "mean_queue_s": float(q.mean()),
        "terms": float(sum(r.terms for r in ok)),
    }
