"""Evidence actors feeding the GPU likelihood scorer.

The reference runs its evidence tasks (generators that suspend on PairHMM
requests) in spawned CPU processes and scores their requests in the parent,
caller/native/caller/gpu_evidence_pipeline.py:74-122.  This module keeps its
message protocol, so the reference's own actor function can run under it:

* parent -> actor: ``("start", identity, task)``, ``("resume", identity,
  likelihoods)`` and ``None`` (stop);
* actor -> parent: ``("request", identity, anchored, pairs)``,
  ``("done", identity, result)`` and ``("error", identity, traceback_text)``.

The scheduling is this module's own:

* every actor has its own command queue and its own response pipe, and the
  parent sleeps in one ``multiprocessing.connection.wait`` over the response
  pipes, the actors' process sentinels (a dead actor is noticed at once) and
  a wake-up pipe written by the scoring thread, so nothing polls;
* a likelihood batch is scored on a background thread (the C-ABI call
  releases the GIL) while the parent keeps serving actors; one batch is in
  flight at a time, since all batches go to the same GPU;
* requests wait in one FIFO per mode (semiglobal, anchored).  A mode is
  flushed as soon as it holds ``max_pairs`` pairs, or when no actor is
  computing (nothing else can arrive before a batch returns); a batch takes
  whole requests from the head of its FIFO up to ``max_pairs`` pairs (a larger
  single request goes alone).
"""
from __future__ import annotations

import collections
import multiprocessing as mp
import traceback
from concurrent.futures import ThreadPoolExecutor
from multiprocessing.connection import wait as wait_for

import numpy as np


class ResponseChannel:
    """The actor's end of its response pipe, with the ``put`` of a queue (what actor
    functions written for a shared ``multiprocessing.Queue`` call)."""

    def __init__(self, connection):
        self.connection = connection

    def put(self, message):
        self.connection.send(message)


def _advance(generator, value, first):
    """Run a task generator to its next request; returns the message for the parent."""
    try:
        anchored, pairs = next(generator) if first else generator.send(value)
    except StopIteration as finished:
        return ("done", finished.value)
    return ("request", bool(anchored), pairs)


def actor(commands, responses, factory):
    """Default actor body: runs the tasks the parent starts as generators made by
    ``factory(task)``.  A generator yields ``(anchored, pairs)`` and is resumed with those
    pairs' ln-likelihoods; its return value is the task's result."""
    live = {}
    current = None
    try:
        for command in iter(commands.get, None):
            kind, current, value = command
            if kind == "start":
                if current in live:
                    raise ValueError(f"task {current} is already running in this actor")
                live[current] = factory(value)
                message = _advance(live[current], None, True)
            elif kind == "resume":
                message = _advance(live[current], value, False)
            else:
                raise ValueError(f"actor command {kind!r} is not start or resume")
            if message[0] == "done":
                live.pop(current)
            responses.put((message[0], current, *message[1:]))
    except BaseException:
        responses.put(("error", current, traceback.format_exc()))
    finally:
        while live:
            live.popitem()[1].close()


def default_scorer():
    from .accelerator import score_pairs
    return lambda pairs, anchored: score_pairs(pairs, anchored=anchored, selection="cuda")


class _Actors:
    """The spawned actor processes and their channels."""

    def __init__(self, count, target, lead, factory):
        ctx = mp.get_context("spawn")
        self.commands = [ctx.Queue() for _ in range(count)]
        pipes = [ctx.Pipe(duplex=False) for _ in range(count)]
        self.inbox = [r for r, _ in pipes]
        self.procs = [ctx.Process(target=target, args=(self.commands[i], ResponseChannel(pipes[i][1]), *lead, factory))
                      for i in range(count)]
        self._senders = [w for _, w in pipes]

    def start(self):
        for p in self.procs:
            p.start()
        for w in self._senders:  # the children hold their own copies
            w.close()

    def send(self, worker, message):
        self.commands[worker].put(message)

    def shutdown(self, clean):
        if clean:
            for q in self.commands:
                q.put(None)
            for p in self.procs:
                p.join(timeout=10)
        for p in self.procs:
            if p.is_alive():
                p.terminate()
                p.join(timeout=5)
        for q in self.commands:
            if not clean:
                q.cancel_join_thread()
            q.close()
        for c in self.inbox:
            c.close()


class _Dispatcher:
    """Parent-side state: live tasks, request FIFOs and the batch on the scoring thread."""

    def __init__(self, tasks, actors, workers, slots, max_pairs, scorer):
        self.tasks = enumerate(tasks)
        self.actors = actors
        self.capacity = workers * slots
        self.max_pairs = max_pairs
        self.scorer = scorer
        self.results = {}
        self.owner = {}                  # identity -> worker
        self.load = [0] * workers        # live tasks per worker
        self.computing = 0               # live tasks whose actor owes a message
        self.fifo = {False: collections.deque(), True: collections.deque()}
        self.queued = {False: 0, True: 0}
        self.batch = None                # (future, [(identity, n_pairs)])
        self.ntasks = 0
        self.pool = ThreadPoolExecutor(max_workers=1, thread_name_prefix="pairhmm-batch")
        self.wake_r, self.wake_w = mp.Pipe(duplex=False)

    # -- tasks ---------------------------------------------------------------
    def admit(self):
        """Start tasks until every actor slot is taken or the task list is exhausted."""
        while len(self.owner) < self.capacity:
            nxt = next(self.tasks, None)
            if nxt is None:
                return
            identity, task = nxt
            self.ntasks = identity + 1
            worker = self.load.index(min(self.load))
            self.owner[identity] = worker
            self.load[worker] += 1
            self.computing += 1
            self.actors.send(worker, ("start", identity, task))

    def on_message(self, worker, message):
        kind, identity, *rest = message
        if kind == "error":
            raise RuntimeError(f"evidence actor {worker} failed:\n{rest[0]}")
        if self.owner.get(identity) != worker:
            raise RuntimeError(f"actor {worker} answered for task {identity}, which it does not own")
        self.computing -= 1
        if kind == "request":
            anchored, pairs = rest
            self.fifo[anchored].append((identity, pairs))
            self.queued[anchored] += len(pairs)
        elif kind == "done":
            self.results[identity] = rest[0]
            del self.owner[identity]
            self.load[worker] -= 1
            self.admit()
        else:
            raise RuntimeError(f"actor {worker} sent a message of unknown kind {kind!r}")

    # -- batches -------------------------------------------------------------
    def maybe_launch(self):
        if self.batch is not None:
            return
        full = [m for m in (False, True) if self.queued[m] >= self.max_pairs]
        if full:
            mode = full[0]
        elif self.computing == 0 and (self.queued[False] or self.queued[True]):
            mode = self.queued[True] > self.queued[False]
        else:
            return
        fifo, taken, count, pairs = self.fifo[mode], [], 0, []
        while fifo and (not taken or count + len(fifo[0][1]) <= self.max_pairs):
            identity, req = fifo.popleft()
            taken.append((identity, len(req)))
            pairs.extend(req)
            count += len(req)
        self.queued[mode] -= count
        fut = self.pool.submit(self.scorer, pairs, mode)
        fut.add_done_callback(lambda _f: self.wake_w.send_bytes(b"."))
        self.batch = (fut, taken)

    def on_batch_done(self):
        fut, taken = self.batch
        self.batch = None
        values = np.asarray(fut.result())
        want = sum(n for _, n in taken)
        if values.ndim != 1 or values.shape[0] != want:
            raise ValueError(f"likelihood scorer returned the wrong shape: {values.shape} for {want} pairs")
        start = 0
        for identity, n in taken:
            self.actors.send(self.owner[identity], ("resume", identity, values[start:start + n]))
            self.computing += 1
            start += n

    # -- loop ----------------------------------------------------------------
    def _read(self, worker, inbox, until_eof=False):
        """Handle the messages waiting on a worker's pipe (after its process ended: all of
        them, up to the end of the pipe).  A worker that is gone while it still owns tasks
        is an error."""
        c = self.actors.inbox[worker]
        try:
            while until_eof or c.poll():
                self.on_message(worker, c.recv())
        except EOFError:
            inbox.pop(c, None)
        if c not in inbox and worker in self.owner.values():
            self.actors.procs[worker].join(timeout=1)
            code = self.actors.procs[worker].exitcode
            raise RuntimeError(f"evidence actor {worker} exited (code {code}) with tasks outstanding")

    def run(self):
        self.admit()
        sentinels = {p.sentinel: i for i, p in enumerate(self.actors.procs)}
        inbox = {c: i for i, c in enumerate(self.actors.inbox)}
        while self.owner:
            self.maybe_launch()
            ready = wait_for([self.wake_r, *inbox, *sentinels])
            if self.wake_r in ready:
                self.wake_r.recv_bytes()
                self.on_batch_done()
            for c in ready:
                if c in inbox:
                    self._read(inbox[c], inbox)
                elif c in sentinels:
                    self._read(sentinels.pop(c), inbox, until_eof=True)
        if self.batch is not None or self.computing or any(self.queued.values()):
            raise RuntimeError("evidence pipeline finished with requests still outstanding")
        return [self.results[i] for i in range(self.ntasks)]

    def close(self):
        self.pool.shutdown(wait=True)
        self.wake_r.close()
        self.wake_w.close()


def run_tasks(tasks, factory, *, workers=4, slots_per_worker=8, max_pairs=32768, scorer=None, actor_target=None,
              actor_args=None):
    """Run ``tasks`` on ``workers`` spawned actors and return their results in task order.

    ``factory(task)`` makes a task's generator.  ``scorer(pairs, anchored) -> float64 array``
    scores one batch (default: this package's ``score_pairs`` on the GPU).  ``actor_target`` /
    ``actor_args`` select the actor function and its leading arguments: it is called as
    ``actor_target(commands, responses, *actor_args, factory)`` in each process (default:
    :func:`actor`), which is the signature of the reference's actor.
    """
    if workers < 1 or slots_per_worker < 1 or max_pairs < 1:
        raise ValueError(f"workers, slots_per_worker and max_pairs must be >= 1 "
                         f"(got {workers}, {slots_per_worker}, {max_pairs})")
    tasks = iter(tasks)
    head = next(tasks, _EMPTY)
    if head is _EMPTY:
        return []
    actors = _Actors(workers, actor_target or actor, tuple(actor_args or ()), factory)
    dispatcher = _Dispatcher(_chain(head, tasks), actors, workers, slots_per_worker, max_pairs,
                             scorer or default_scorer())
    clean = False
    try:
        actors.start()
        results = dispatcher.run()
        clean = True
        return results
    finally:
        dispatcher.close()
        actors.shutdown(clean)


_EMPTY = object()


def _chain(head, rest):
    yield head
    yield from rest
