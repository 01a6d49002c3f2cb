"""The autotuner's table as text (no GPU needed): load, save, round trip,
and a malformed file rejected."""
import pytest

from statfem_b200 import api


def test_cache_round_trip(tmp_path):
    api.autotune_clear()
    p = tmp_path / "tune.txt"
    p.write_text("# comment\nblock:NVIDIA_B200/sm148:n18:d3:r78:k8 128 1\nspmv:NVIDIA_B200/sm148:n18:d3:r78:k0 32\n")
    api.autotune_load(p)
    q = tmp_path / "out.txt"
    api.autotune_save(q)
    lines = [l for l in q.read_text().splitlines() if not l.startswith("#")]
    assert sorted(lines) == sorted(["block:NVIDIA_B200/sm148:n18:d3:r78:k8 128 1",
                                    "spmv:NVIDIA_B200/sm148:n18:d3:r78:k0 32"])
    api.autotune_clear()


def test_cache_rejects_malformed(tmp_path):
    p = tmp_path / "bad.txt"
    p.write_text("no-value-on-this-line\n")
    with pytest.raises(api.SfcError):
        api.autotune_load(p)
    with pytest.raises(api.SfcError):
        api.autotune_load(tmp_path / "missing.txt")
    api.autotune_clear()
