"""Host logic of the batch autotuner (dba_b200/autotune.py) on the CPU: the
fastest (block edge, threads) pair is chosen, the chunk keeps the mean overshoot
past a stop within 5 % of the shortest sweep run, and the choice is cached per
device and precision.  The timing of each candidate is replaced by known scores."""
import json

from dba_b200 import autotune


class FakeDevice:
    """Stands in for torch.cuda on a host without a GPU: two devices, one current."""
    names = {0: ("NVIDIA B200", 10, 0, 148), 1: ("Other GPU", 9, 0, 132)}

    def __init__(self):
        self.cur = 0

    def current_device(self):
        return self.cur

    def get_device_properties(self, d):
        from types import SimpleNamespace
        n, ma, mi, sms = self.names[d]
        return SimpleNamespace(name=n, major=ma, minor=mi, multi_processor_count=sms)


def _fake_torch(monkeypatch):
    import sys
    from types import SimpleNamespace
    dev = FakeDevice()
    monkeypatch.setitem(sys.modules, "torch", SimpleNamespace(cuda=dev))
    return dev


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
    cache = tmp_path / "autotune.json"
    monkeypatch.setenv("DBA_AUTOTUNE_CACHE", str(cache))
    _fake_torch(monkeypatch)
    scores = {(8, 128): 1.0, (8, 256): 3.0, (8, 512): 2.0, (16, 128): 0.5, (16, 256): 2.5, (16, 512): 2.9}
    calls = []

    def fake_time(block, threads=256, precision=1, persistent=1, **kw):
        calls.append((block, threads, precision, persistent))
        # the per-step form wins for block 8 threads 256 only
        return scores[(block, threads)] + (0.1 if (block, threads, persistent) == (8, 256, 0) else 0.0)

    monkeypatch.setattr(autotune, "time_candidate", fake_time)
    c = autotune.tune(precision=1, use_cache=True)
    assert (c["block"], c["threads"], c["persistent"]) == (8, 256, 0)
    assert c["chunk"] == 96 and c["chunk"] / 2 <= 0.05 * autotune.SHORTEST_RUN_STEPS
    assert len(calls) == 2 * len(scores)
    stored = json.load(open(cache))
    assert list(stored.values())[0]["block"] == 8
    # cached: no new timing runs
    c2 = autotune.tune(precision=1, use_cache=True)
    assert len(calls) == 2 * len(scores) and (c2["block"], c2["threads"]) == (8, 256)
    # other precision: a separate entry
    autotune.tune(precision=0, use_cache=True)
    assert len(calls) == 4 * len(scores) and len(json.load(open(cache))) == 2


def test_cache_key_follows_the_current_device(tmp_path, monkeypatch):
    """Each GPU gets its own entry: the key is built from the current device's
    properties, not from device 0 or a shared constant."""
    cache = tmp_path / "autotune.json"
    monkeypatch.setenv("DBA_AUTOTUNE_CACHE", str(cache))
    dev = _fake_torch(monkeypatch)
    calls = []

    def fake_time(block, threads=256, precision=1, persistent=1, **kw):
        calls.append(dev.cur)
        return float(block * threads) if dev.cur == 0 else float(1000 - block * threads)

    monkeypatch.setattr(autotune, "time_candidate", fake_time)
    a = autotune.tune(precision=1, use_cache=True)
    dev.cur = 1
    b = autotune.tune(precision=1, use_cache=True)
    assert (a["block"], a["threads"]) == (16, 512) and (b["block"], b["threads"]) == (8, 128)
    keys = sorted(json.load(open(cache)))
    assert len(keys) == 2 and any("B200" in k for k in keys) and any("Other GPU" in k for k in keys)
    n = len(calls)
    dev.cur = 0
    assert (autotune.tune(precision=1, use_cache=True)["block"]) == 16 and len(calls) == n   # served from the cache


def test_tune_without_cache_leaves_no_file(tmp_path, monkeypatch):
    cache = tmp_path / "none.json"
    monkeypatch.setenv("DBA_AUTOTUNE_CACHE", str(cache))
    _fake_torch(monkeypatch)
    monkeypatch.setattr(autotune, "time_candidate",
                        lambda block, threads=256, precision=1, persistent=1, **kw: block * threads + persistent)
    c = autotune.tune(precision=1, use_cache=False)
    assert (c["block"], c["threads"]) == (16, 512)
    assert not cache.exists()
