"""Per-call device timing of the C ABI (CUDA events) and NVTX ranges.

``with Timeline() as tl: ...`` records a CUDA event pair on the current stream
around every library entry point called inside the block (``_lib.call``);
``tl.summary()`` then gives, per entry point, the number of calls and their total
and mean device time in milliseconds.  Events are read only when the summary is
asked for, so timing does not add host synchronisation.  ``Timeline(all_threads=True)``
also records calls made by other threads meanwhile (torch's autograd engine runs the
backward passes of CUDA tensors on its own thread).
"""
import threading
from collections import defaultdict

_state = threading.local()
_shared = {'timeline': None}


def active():
    return getattr(_state, 'timeline', None) or _shared['timeline']


class Timeline:

    def __init__(self, nvtx=False, all_threads=False):
        self.records = []
        self.nvtx = nvtx
        self.all_threads = all_threads

    def __enter__(self):
        self._prev = getattr(_state, 'timeline', None)
        _state.timeline = self
        if self.all_threads:
            self._prev_shared = _shared['timeline']
            _shared['timeline'] = self
        return self

    def __exit__(self, *exc):
        _state.timeline = self._prev
        if self.all_threads:
            _shared['timeline'] = self._prev_shared

    def start(self, name):
        import torch
        if self.nvtx:
            torch.cuda.nvtx.range_push(name)
        begin = torch.cuda.Event(enable_timing=True)
        begin.record()
        return name, begin

    def stop(self, token):
        import torch
        name, begin = token
        end = torch.cuda.Event(enable_timing=True)
        end.record()
        if self.nvtx:
            torch.cuda.nvtx.range_pop()
        self.records.append((name, begin, end))

    def summary(self):
        import torch
        torch.cuda.synchronize()
        out = defaultdict(lambda: {'calls': 0, 'total_ms': 0.})
        for name, begin, end in self.records:
            out[name]['calls'] += 1
            out[name]['total_ms'] += begin.elapsed_time(end)
        for v in out.values():
            v['mean_ms'] = v['total_ms'] / max(v['calls'], 1)
        return dict(out)
