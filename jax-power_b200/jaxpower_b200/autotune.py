"""Autotuner for the paint tile configuration (tile shape / CTA size).

``best_tile_config(key, run)`` times ``run(config)`` for every tile configuration of
``pk_paint_batch`` with CUDA events (after one warm-up call each) and returns the
fastest; results are cached in memory and in a JSON file (``$JAXPOWER_B200_AUTOTUNE`` or
``~/.cache/jaxpower_b200/autotune.json``) keyed by GPU name and the caller's key (mesh
size, resampler, interlacing, particle-count bucket).  ``PK_AUTOTUNE=0`` disables
tuning (configuration 0 is used).
"""
import json
import os
import threading

import torch

NUM_TILE_CONFIGS = 11
_cache = {}
_lock = threading.Lock()


def _path():
    return os.environ.get('JAXPOWER_B200_AUTOTUNE',
                          os.path.join(os.path.expanduser('~'), '.cache', 'jaxpower_b200', 'autotune.json'))


def _load():
    try:
        with open(_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table):
    path = _path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + '.tmp'
        with open(tmp, 'w') as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def make_key(*parts):
    return '|'.join([torch.cuda.get_device_name()] + [str(p) for p in parts])


def cached_tile_config(key, default=0):
    """The tuned configuration of ``key`` when there is one (memory or file), else ``default``."""
    with _lock:
        if key in _cache:
            return _cache[key]
        table = _load()
        if key in table:
            _cache[key] = int(table[key]['config'])
            return _cache[key]
    return default


def best_tile_config(key, run, repeats=3):
    """Fastest tile configuration for ``key``; ``run(config)`` enqueues one paint."""
    if os.environ.get('PK_AUTOTUNE', '1') == '0':
        return 0
    with _lock:
        if key in _cache:
            return _cache[key]
        table = _load()
        if key in table:
            _cache[key] = int(table[key]['config'])
            return _cache[key]
    times = {}
    for config in range(NUM_TILE_CONFIGS):
        run(config)  # warm-up (and kernel attribute set-up)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(repeats):
            run(config)
        end.record()
        torch.cuda.synchronize()
        times[config] = start.elapsed_time(end) / repeats
    best = min(times, key=times.get)
    with _lock:
        _cache[key] = best
        table = _load()
        table[key] = {'config': best, 'ms': {str(k): round(v, 4) for k, v in times.items()}}
        _store(table)
    return best
