"""Evidence actors feeding the GPU: the parent-side loop of
caller/native/caller/gpu_evidence_pipeline.py:74-122 with the likelihood
batches scored asynchronously.

The reference's actors (spawned CPU processes) run generator tasks that yield
lists of (read, qualities, haplotype) PairHMM requests and are resumed with
the likelihoods; the parent gathers the requests of all actors into batches of
up to ``max_pairs`` pairs of one mode (semiglobal or anchored) and scores each
batch in one call.  There the parent stops collecting while a batch scores.
Here the batch goes to a scoring thread (the C ABI call releases the GIL, the
packing and the kernels run off the parent loop) and the parent keeps
draining actor messages and starting tasks meanwhile; when the batch
completes its likelihoods are sent back in the same order.  The message
protocol, the batch selection rule and the error behaviour are the
reference's, so its own actor function can run under this loop
(``actor=gpu_evidence_pipeline._actor`` with ``actor_args=(arguments,
reference)``).
"""
from __future__ import annotations

import itertools
import multiprocessing as mp
import queue
import traceback
from concurrent.futures import ThreadPoolExecutor

import numpy as np


def actor(commands, responses, factory):
    """A worker process: runs generator tasks made by ``factory(payload)``; every value a task
    yields is ``(anchored, requests)`` and it is resumed with the requests' likelihoods."""
    sessions = {}
    identity = None
    try:
        while True:
            command = commands.get()
            if command is None:
                return
            kind, identity, payload = command
            if kind == "start":
                if identity in sessions:
                    raise ValueError("Duplicate active evidence task")
                generator = factory(payload)
                sessions[identity] = generator
                first = True
            elif kind == "resume":
                generator = sessions[identity]
                first = False
            else:
                raise ValueError("Unknown evidence actor command")
            try:
                anchored, requests = next(generator) if first else generator.send(payload)
                responses.put(("request", identity, bool(anchored), requests))
            except StopIteration as done:
                del sessions[identity]
                responses.put(("done", identity, done.value))
    except BaseException:
        responses.put(("error", identity, traceback.format_exc()))
    finally:
        for generator in sessions.values():
            generator.close()


def default_scorer():
    from .accelerator import score_pairs
    return lambda requests, anchored: score_pairs(requests, anchored=anchored, selection="cuda")


def run_tasks(tasks, factory, *, workers=4, slots_per_worker=8, max_pairs=32768, scorer=None, actor_target=None,
              actor_args=None, poll=0.05):
    """Run ``tasks`` on ``workers`` spawned actors and return their results in task order.

    ``scorer(requests, anchored) -> float64 array`` scores one batch (default: this package's
    score_pairs on the GPU).  ``actor_target``/``actor_args`` select the worker function and its
    leading arguments (default: ``actor`` above, called as actor(commands, responses, factory)).
    """
    if workers < 1 or slots_per_worker < 1 or max_pairs < 1:
        raise ValueError("Invalid evidence pipeline bounds")
    scorer = scorer or default_scorer()
    target = actor_target or actor
    lead = tuple(actor_args or ())
    tasks = iter(tasks)
    try:
        first = next(tasks)
    except StopIteration:
        return []
    tasks = itertools.chain([first], tasks)
    context = mp.get_context("spawn")
    window = workers * slots_per_worker
    responses = context.Queue(maxsize=2 * window)
    commands = [context.Queue(maxsize=2 * slots_per_worker) for _ in range(workers)]
    processes = [context.Process(target=target, args=(commands[i], responses, *lead, factory))
                 for i in range(workers)]
    owners, loads, results, pending = {}, [0] * workers, [], []
    inflight = 0
    exhausted = False
    success = False
    batch = None  # (future, selected) of the batch being scored
    pool = ThreadPoolExecutor(max_workers=1)

    def fill():
        nonlocal exhausted, inflight
        while not exhausted and len(owners) < window:
            try:
                task = next(tasks)
            except StopIteration:
                exhausted = True
                break
            worker = min(range(workers), key=lambda i: loads[i])
            identity = len(results)
            results.append(None)
            owners[identity] = worker
            loads[worker] += 1
            commands[worker].put(("start", identity, task))
            inflight += 1

    def finish(fut, selected):
        nonlocal inflight
        values = np.asarray(fut.result())
        count = sum(len(x[2]) for x in selected)
        if values.ndim != 1 or len(values) != count:
            raise ValueError("Likelihood scorer returned the wrong shape")
        offset = 0
        for identity, _, jobs in selected:
            commands[owners[identity]].put(("resume", identity, values[offset:offset + len(jobs)]))
            offset += len(jobs)
            inflight += 1

    try:
        for process in processes:
            process.start()
        fill()
        while owners:
            # with no actor computing nothing else can arrive: wait for the batch
            if batch is not None and (batch[0].done() or inflight == 0):
                fut, selected = batch
                batch = None
                finish(fut, selected)
                continue
            if batch is None and pending and (inflight == 0 or sum(len(x[2]) for x in pending) >= max_pairs):
                # the reference's selection: the first pending mode, up to max_pairs pairs
                mode = pending[0][1]
                selected, rest, count = [], [], 0
                for item in pending:
                    if item[1] == mode and (not selected or count + len(item[2]) <= max_pairs):
                        selected.append(item)
                        count += len(item[2])
                    else:
                        rest.append(item)
                pending = rest
                requests = [p for _, _, jobs in selected for p in jobs]
                batch = (pool.submit(scorer, requests, mode), selected)
                continue
            try:
                message = responses.get(timeout=poll if batch is not None else 2)
            except queue.Empty:
                if any(not p.is_alive() for p in processes):
                    raise RuntimeError("Evidence worker exited before completing its tasks")
                continue
            kind, identity, *payload = message
            if kind == "error":
                raise RuntimeError("Evidence worker failed:\n" + payload[0])
            if identity not in owners:
                raise RuntimeError("Unowned evidence response")
            inflight -= 1
            if kind == "request":
                pending.append((identity, *payload))
            elif kind == "done":
                results[identity] = payload[0]
                loads[owners.pop(identity)] -= 1
                fill()
            else:
                raise RuntimeError("Unknown evidence response")
        if pending or inflight or batch is not None:
            raise RuntimeError("Evidence accounting mismatch")
        success = True
        return results
    finally:
        pool.shutdown(wait=True)
        if success:
            for q in commands:
                q.put(None)
            for p in processes:
                p.join(timeout=10)
        for p in processes:
            if p.is_alive():
                p.terminate()
                p.join(timeout=2)
        for q in [*commands, responses]:
            if not success:
                q.cancel_join_thread()
