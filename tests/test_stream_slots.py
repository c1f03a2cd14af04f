'''The scheduling of the streamed fit (analysis/_fit.py, fit_stream) on
host jobs, no GPU: at most ``depth`` jobs run at once on distinct slots, a
slot frees when ANY job ends (a slow batch does not hold back the ones
behind it), results leave in submission order, empty batches pass through
in their place, and the finished backlog stays bounded.'''
import threading
from concurrent.futures import ThreadPoolExecutor

import pytest

from pylorenzmie_b200.analysis._fit import _Slots


class _Jobs:
    '''Fake fits: job i runs gate(i) and returns (i, slot).'''

    def __init__(self, depth):
        self.pool = ThreadPoolExecutor(max_workers=depth + 2)
        self.lock = threading.Lock()
        self.running = {}
        self.most = 0
        self.started = {}
        self.clash = False

    def launch(self, slot, i, gate):
        def job():
            with self.lock:
                self.clash |= slot in self.running.values()
                self.running[i] = slot
                self.most = max(self.most, len(self.running))
                self.started[i] = threading.Event()
                self.started[i].set()
            try:
                gate(i)
            finally:
                with self.lock:
                    del self.running[i]
            return i, slot
        return self.pool.submit(job)


def _run(slots, jobs, plan, gate):
    '''fit_stream's loop over ``plan`` (True: a batch with a fit, False: an
    empty one); returns what it yields, in order, and the largest number
    of entries queued.'''
    out, most_pending = [], 0
    for i, has_fit in enumerate(plan):
        if not has_fit:
            slots.add_done(('empty', i))
            continue
        slots.wait_slot()
        out.extend(slots.ready())
        slots.submit(jobs.launch, ('batch', i), i, gate)
        most_pending = max(most_pending, len(slots.pending))
    out.extend(slots.drain())
    slots.wait_all()
    return out, most_pending


@pytest.mark.parametrize('depth', [1, 2, 4])
def test_order_and_concurrency(depth):
    jobs = _Jobs(depth)
    slots = _Slots(depth)
    plan = [True, True, False, True, True, True, False, False, True] * 3
    out, _ = _run(slots, jobs, plan, lambda i: None)
    assert len(out) == len(plan)
    for i, (entry, has_fit) in enumerate(zip(out, plan)):
        if has_fit:
            got_i, slot, extra = entry
            assert got_i == i and extra == ('batch', i) and 0 <= slot < depth
        else:
            assert entry == ('empty', i)
    assert jobs.most <= depth and not jobs.clash
    assert sorted(slots.free + list(slots.running.values())) == \
        list(range(depth))


def test_a_slow_batch_holds_one_slot_only():
    '''Depth 2: batch 0 runs until batch 6 has started; the batches between
    pass through the other slot meanwhile (with oldest-first freeing the
    loop would wait on batch 0 and batch 6 would never start: the gate
    would time out).'''
    depth = 2
    jobs = _Jobs(depth)
    slots = _Slots(depth)
    seen = {}

    def gate(i):
        if i == 0:
            ok = False
            for _ in range(200):         # bounded: 10 s at most
                with jobs.lock:
                    ev = jobs.started.get(6)
                if ev is not None:
                    ok = True
                    break
                threading.Event().wait(0.05)
            seen['batch 6 started while batch 0 ran'] = ok
    out, _ = _run(slots, jobs, [True] * 8, gate)
    assert seen['batch 6 started while batch 0 ran']
    assert [e[0] for e in out] == list(range(8))
    assert jobs.most <= depth and not jobs.clash


def test_backlog_is_bounded():
    '''Batch 0 is slow; the finished batches behind it queue up to the
    backlog bound, past which the oldest is waited for and yielded.'''
    depth, backlog = 2, 5
    jobs = _Jobs(depth)
    slots = _Slots(depth, backlog=backlog)
    release = threading.Event()

    def gate(i):
        if i == 0:
            release.wait(0.5)
    out, most_pending = _run(slots, jobs, [True] * 20, gate)
    assert most_pending <= backlog
    assert [e[0] for e in out] == list(range(20))
    assert _Slots(3).backlog == 24
