"""The autotuner's cache on the CPU: a configuration stored for a key is applied
to the decoder without timing anything, for single- and multi-instance
decoders, and other keys in the same file are left alone."""
import json
import types

from brkga_fft2_b200.autotune import autotune


class FakeDecoder:
    def __init__(self, multi=False):
        self.calls = []
        self.device = types.SimpleNamespace(index=0)
        if multi:
            self.packs = ["a", "b"]
        else:
            self.packed = "a"

    def set_launch_config(self, *cfg):
        self.calls.append(cfg)


def test_cached_configuration_is_applied_without_timing(tmp_path):
    path = tmp_path / "tune.json"
    cache = {"dev|grid300x300": {"config": [2, 16, 0, 1024], "ms": 3.5, "table": [[2, 16, 0, -1, 3.6]]},
             "other": {"config": [4, 8, 1, 8192], "ms": 1.0, "table": []}}
    path.write_text(json.dumps(cache))
    for multi in (False, True):
        dec = FakeDecoder(multi)
        res = autotune(dec, chrom=None, key="dev|grid300x300", cache_path=str(path))
        assert res["cached"] and res["config"] == (2, 16, 0, 1024) and res["ms"] == 3.5
        assert dec.calls == [(2, 16, 0, 1024)]
    assert json.loads(path.read_text()) == cache  # a cache hit does not rewrite the file
