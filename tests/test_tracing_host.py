"""The C-ABI call timeline on the CPU: ``_lib.call`` brackets every entry point called inside
a ``tracing.Timeline`` with an event pair (CUDA events replaced by a fake clock here; the calls
are host-only workspace queries and argument errors), failing calls included, and the summary
counts calls and device time per entry point.  Timelines nest and ``all_threads`` sees calls
from other threads."""
import ctypes
import threading

import pytest


@pytest.fixture
def fake_events(monkeypatch):
    import torch
    clock = {'now': 0.}

    class Event:
        def __init__(self, enable_timing=False):
            self.t = None

        def record(self, stream=None):
            clock['now'] += 1.
            self.t = clock['now']

        def elapsed_time(self, end):
            return end.t - self.t

    monkeypatch.setattr(torch.cuda, 'Event', Event)
    monkeypatch.setattr(torch.cuda, 'synchronize', lambda *a, **k: None)
    return clock


def _query(L):
    nbytes = L.c_size_t()
    L.call('pk_paint_workspace_size', 1000, L.i32([64, 64, 64]), 3, 3, ctypes.byref(nbytes))
    return nbytes.value


def test_timeline_counts_calls(fake_events):
    from jaxpower_b200 import _lib as L
    from jaxpower_b200.tracing import Timeline, active
    assert active() is None
    with Timeline() as outer:
        assert _query(L) > 0
        with Timeline() as inner:
            _query(L)
            with pytest.raises(L.PKError):  # order 5: an argument error, still timed
                L.call('pk_paint_workspace_size', 1000, L.i32([64, 64, 64]), 5, 3, ctypes.byref(L.c_size_t()))
        assert active() is outer
        _query(L)
    assert active() is None
    s = inner.summary()
    assert s['pk_paint_workspace_size']['calls'] == 2
    assert s['pk_paint_workspace_size']['total_ms'] == pytest.approx(2.)  # one tick per call
    s = outer.summary()
    assert s['pk_paint_workspace_size']['calls'] == 2
    assert s['pk_paint_workspace_size']['mean_ms'] == pytest.approx(1.)
    _query(L)  # outside any timeline: nothing recorded
    assert len(outer.records) == 2


def test_timeline_all_threads(fake_events):
    from jaxpower_b200 import _lib as L
    from jaxpower_b200.tracing import Timeline
    L.load()
    with Timeline(all_threads=True) as tl:
        t = threading.Thread(target=_query, args=(L,))
        t.start()
        t.join()
    with Timeline() as local:
        t = threading.Thread(target=_query, args=(L,))
        t.start()
        t.join()
    assert tl.summary()['pk_paint_workspace_size']['calls'] == 1
    assert local.summary() == {}
