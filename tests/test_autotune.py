"""Autotuner: candidates, size buckets, the JSON cache, and (GPU) that block size leaves results
bit-identical while the tuner returns one of its candidates."""
import numpy as np
import pytest

from epp import abi, autotune, casegen


def test_candidates_and_buckets():
    c = autotune.candidates()
    assert (0, 128) in c and (0, 64) in c and (0, 32) in c and (4, 128) in c
    assert all(f == 0 for f, _ in autotune.candidates(batch=True))
    assert autotune.size_bucket(1000) == 12 and autotune.size_bucket(10**6) == 24
    assert autotune.size_bucket(3000) == autotune.size_bucket(3100)


def test_cache_roundtrip_and_reuse(tmp_path, monkeypatch):
    path = str(tmp_path / "tune.json")
    calls = []

    def fake_tune(case, steps=20, device=0, batch=None, **kw):
        calls.append(case)
        return (4, 128), {(0, 128): 2.0, (4, 128): 1.0}

    monkeypatch.setattr(autotune, "tune_case", fake_tune)
    monkeypatch.setattr(autotune, "representative_case", lambda dim, n: type("C", (), {"n": n})())
    t = autotune.Autotuner(cache=autotune.TuneCache(path), gpu="B200")
    assert t.best(2, 5000) == (4, 128)
    assert t.best(2, 5200) == (4, 128)          # same bucket: cached
    assert len(calls) == 1
    again = autotune.Autotuner(cache=autotune.TuneCache(path), gpu="B200")
    assert again.best(2, 5000) == (4, 128)      # persisted
    assert len(calls) == 1
    key = autotune.TuneCache.key("B200", 2, 5000, False)
    assert again.cache.get(key)["ms_per_step"]["4/128"] == 1.0


def test_concurrent_mode_keys():
    """Serving tunes for throughput with several runs resident: its own cache entries, and
    fewer copies of large runs."""
    assert autotune.TuneCache.key("B200", 2, 5000, False, 16).endswith("|concurrent16")
    assert autotune.TuneCache.key("B200", 2, 5000, False, 1).endswith("|single")
    assert autotune.TuneCache.key("B200", 2, 5000, True, 16).endswith("|batch")
    assert autotune.concurrent_copies(3e4) == 16
    assert autotune.concurrent_copies(1e6) == 4
    assert autotune.concurrent_copies(1e8) == 1


@pytest.mark.gpu
def test_tune_concurrent_small_case():
    case = casegen.dam_break_2d(dx=0.05, max_neighbour_number=1)
    best, ms = autotune.tune_case(case, steps=3, concurrent=3)
    assert best in autotune.candidates()
    assert set(ms) == set(autotune.candidates()) and all(v > 0 for v in ms.values())


@pytest.mark.gpu
def test_block_threads_bit_identical():
    outs = []
    for thr in (128, 64, 32):
        case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
        from epp.algorithm import DeviceParticleSystem
        from epp.classes import NeighbourSystem
        ns = NeighbourSystem(case.domain, casegen.DAM_BREAK_ACTIVE_PAIRS, max_neighbour_number=1)
        d = DeviceParticleSystem(case.ps, ns)
        d.ctx.set_block_threads(thr)
        d.syncto()
        d.ctx.search(abi.EPP_CRITERION_SYMMETRY, abi.EPP_ACTION_DAMBREAK_CONTINUITY, case.physics, 0)
        d.ctx.step(20, case.physics)
        d.asyncto()
        outs.append({k: d.host[k] for k in ("PositionVec", "VelocityVec", "Density", "nCount")})
        d.close()
    for o in outs[1:]:
        for k in o:
            assert np.array_equal(o[k], outs[0][k]), k


@pytest.mark.gpu
def test_tune_small_case(tmp_path):
    case = casegen.dam_break_2d(dx=0.04, max_neighbour_number=1)
    best, ms = autotune.tune_case(case, steps=5)
    assert best in autotune.candidates()
    assert set(ms) == set(autotune.candidates()) and all(v > 0 for v in ms.values())
    t = autotune.Autotuner(cache=autotune.TuneCache(str(tmp_path / "t.json")), steps=5)
    assert t.best(2, case.n, case=case) in autotune.candidates()
