"""Per-call device timing of the C ABI (CUDA events) and NVTX ranges.

``with Timeline() as tl: ...`` records a CUDA event pair on the current stream
around every library entry point called inside the block (``_lib.call``);
``tl.summary()`` then gives, per entry point, the number of calls and their total
and mean device time in milliseconds.  Events are read only when the summary is
asked for, so timing does not add host synchronisation.
"""
import threading
from collections import defaultdict

_state = threading.local()


def active():
    return getattr(_state, 'timeline', None)


class Timeline:

    def __init__(self, nvtx=False):
        self.records = []
        self.nvtx = nvtx

    def __enter__(self):
        self._prev = active()
        _state.timeline = self
        return self

    def __exit__(self, *exc):
        _state.timeline = self._prev

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
