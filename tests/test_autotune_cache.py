"""The autotuner's cache logic on CPU, with a stand-in for the context."""
import json

from fluid_step import _abi
from fluid_step.autotune import cache_key, load_cache, tune


class FakeData:
    count = 1 << 20
    table_size = 1 << 20

    def __init__(self):
        self.applied = None
        self.measured = 0

    def set_tuning(self, t):
        self.applied = (t.radix_digit_bits, t.radix_items, t.mlp_ctas_per_sm,
                        list(t.nbr_threads), list(t.nbr_persistent))

    def autotune(self):
        self.measured += 1
        r = _abi.FeTuneReport()
        r.radix_candidates = 2
        r.radix_digit_bits[0], r.radix_items[0], r.radix_ms[0] = 8, 16, 0.2
        r.radix_digit_bits[1], r.radix_items[1], r.radix_ms[1] = 10, 8, 0.1
        r.chosen = _abi.FeTuning(10, 8, 4, 0)
        r.chosen.nbr_threads[:] = [128, 512, 256, 256]
        r.chosen.nbr_persistent[:] = [0, 1, 1, 0]
        return r


def test_measures_then_reuses(tmp_path):
    path = str(tmp_path / "tune.json")
    d = FakeData()
    r1 = tune(d, path, device="B200|sm148")
    assert r1["source"] == "measured" and d.measured == 1
    assert r1["tuning"] == {"radix_digit_bits": 10, "radix_items": 8, "mlp_ctas_per_sm": 4,
                            "nbr_threads": [128, 512, 256, 256],
                            "nbr_persistent": [0, 1, 1, 0]}
    assert len(r1["report"]["radix"]) == 2
    d2 = FakeData()
    r2 = tune(d2, path, device="B200|sm148")
    assert r2["source"] == "cache" and d2.measured == 0
    assert d2.applied == (10, 8, 4, [128, 512, 256, 256], [0, 1, 1, 0])


def test_cache_entries_without_neighbour_shapes_apply_the_defaults(tmp_path):
    path = tmp_path / "old.json"
    key = cache_key("B200|sm148", FakeData.count, FakeData.table_size, False)
    path.write_text(json.dumps({key: {"radix_digit_bits": 8, "radix_items": 16,
                                      "mlp_ctas_per_sm": 3}}))
    d = FakeData()
    r = tune(d, str(path), device="B200|sm148")
    assert r["source"] == "cache"
    assert d.applied == (8, 16, 3, [256] * 4, [0] * 4)


def test_key_separates_classes():
    a = cache_key("B200|sm148", 1 << 20, 1 << 20, False)
    assert a != cache_key("B200|sm148", 1 << 20, 1 << 20, True)
    assert a != cache_key("B200|sm148", 1 << 18, 1 << 18, False)
    assert a != cache_key("H100|sm132", 1 << 20, 1 << 20, False)
    assert a == cache_key("B200|sm148", (1 << 20) - 5, 1 << 20, False)


def test_unreadable_cache_is_empty(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text("{not json")
    assert load_cache(str(p)) == {}
    p.write_text(json.dumps([1, 2]))
    assert load_cache(str(p)) == {}
    assert load_cache(None) == {}
