"""The paint-tile autotuner's host logic on the CPU, with CUDA events replaced by a fake clock:
it picks the fastest configuration, stores it in its JSON table, serves it from memory and
from the file afterwards, and ``PK_AUTOTUNE=0`` turns tuning off."""
import json

import pytest


class _Clock:
    """Fake device clock: run(config) advances it by that configuration's cost."""

    def __init__(self, costs):
        self.now, self.costs, self.calls = 0., costs, []

    def run(self, config):
        self.calls.append(config)
        self.now += self.costs[config]


def _fake_cuda(monkeypatch, clock):
    import torch

    class Event:
        def __init__(self, enable_timing=False):
            self.t = None

        def record(self, stream=None):
            self.t = clock.now

        def elapsed_time(self, end):
            return end.t - self.t

    monkeypatch.setattr(torch.cuda, 'Event', Event)
    monkeypatch.setattr(torch.cuda, 'synchronize', lambda *a, **k: None)


@pytest.fixture
def tuner(monkeypatch, tmp_path):
    from jaxpower_b200 import autotune
    monkeypatch.setenv('JAXPOWER_B200_AUTOTUNE', str(tmp_path / 'autotune.json'))
    monkeypatch.delenv('PK_AUTOTUNE', raising=False)
    monkeypatch.setattr(autotune, '_cache', {})
    return autotune


def test_picks_fastest_and_persists(monkeypatch, tuner, tmp_path):
    costs = {c: 1. + 0.1 * ((7 * c) % tuner.NUM_TILE_CONFIGS) for c in range(tuner.NUM_TILE_CONFIGS)}
    costs[9] = 0.25
    clock = _Clock(costs)
    _fake_cuda(monkeypatch, clock)
    key = 'B200|paint|(512, 512, 512)|3|3|44'
    assert tuner.best_tile_config(key, clock.run, repeats=3) == 9
    # every configuration: one warm-up call and `repeats` timed ones
    assert sorted(set(clock.calls)) == list(range(tuner.NUM_TILE_CONFIGS))
    assert len(clock.calls) == 4 * tuner.NUM_TILE_CONFIGS
    table = json.loads((tmp_path / 'autotune.json').read_text())
    assert table[key]['config'] == 9
    assert table[key]['ms']['9'] == pytest.approx(0.25)
    # from memory: nothing runs again
    clock.calls.clear()
    assert tuner.best_tile_config(key, clock.run) == 9 and clock.calls == []
    # from the file, in a fresh process-level cache
    monkeypatch.setattr(tuner, '_cache', {})
    assert tuner.cached_tile_config(key, default=0) == 9
    monkeypatch.setattr(tuner, '_cache', {})
    assert tuner.best_tile_config(key, clock.run) == 9 and clock.calls == []
    assert tuner.cached_tile_config('another key', default=4) == 4


def test_tuning_off(monkeypatch, tuner):
    clock = _Clock({c: 1. for c in range(tuner.NUM_TILE_CONFIGS)})
    _fake_cuda(monkeypatch, clock)
    monkeypatch.setenv('PK_AUTOTUNE', '0')
    assert tuner.best_tile_config('k', clock.run) == 0 and clock.calls == []


def test_unreadable_table_is_ignored(monkeypatch, tuner, tmp_path):
    (tmp_path / 'autotune.json').write_text('{not json')
    clock = _Clock({c: 2. - 0.1 * c for c in range(tuner.NUM_TILE_CONFIGS)})
    _fake_cuda(monkeypatch, clock)
    best = tuner.NUM_TILE_CONFIGS - 1
    assert tuner.best_tile_config('k', clock.run) == best
    assert json.loads((tmp_path / 'autotune.json').read_text())['k']['config'] == best
