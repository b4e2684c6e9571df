"""Host logic of the first-point estimator: how (ell, m) terms are grouped into transforms.

Whole ells (every m, in order) stay together whenever they fit, so that the compiled
whole-ell kernels take them; an ell larger than a batch is split (general kernels).
"""
import pytest

from jaxpower_b200 import mesh2


def _batches(monkeypatch, ells, batch):
    monkeypatch.setattr(mesh2, '_term_batch', lambda mattrs, nterms: min(nterms, batch))
    return mesh2._term_batches(None, ells)


def _ells_of(batch):
    return sorted({ell for ell, _ in batch})


@pytest.mark.parametrize('batch', [32, 14, 13, 9, 5])
def test_whole_ells_grouped(monkeypatch, batch):
    out = _batches(monkeypatch, (0, 2, 4), batch)
    flat = [t for b in out for t in b]
    assert flat == [(2, m) for m in range(-2, 3)] + [(4, m) for m in range(-4, 5)]
    assert all(len(b) <= batch for b in out)
    if batch >= 9:  # every batch is made of whole ells
        for b in out:
            for ell in _ells_of(b):
                assert [t for t in b if t[0] == ell] == [(ell, m) for m in range(-ell, ell + 1)]
        assert len(out) == (1 if batch >= 14 else 2)
    else:  # ell 4 (9 terms) is split, ell 2 stays whole
        assert out[0] == [(2, m) for m in range(-2, 3)]


def test_unsorted_ells_and_odd(monkeypatch):
    out = _batches(monkeypatch, (4, 0, 1, 3, 2), 32)
    assert [t[0] for t in out[0]] == [1] * 3 + [2] * 5 + [3] * 7 + [4] * 9


def test_ell_larger_than_batch_is_split(monkeypatch):
    out = _batches(monkeypatch, (0, 2, 8), 6)
    flat = [t for b in out for t in b]
    assert flat == [(2, m) for m in range(-2, 3)] + [(8, m) for m in range(-8, 9)]
    assert all(len(b) <= 6 for b in out)
    assert out[0] == [(2, m) for m in range(-2, 3)]


def test_monopole_only(monkeypatch):
    assert _batches(monkeypatch, (0,), 8) == []
