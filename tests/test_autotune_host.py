"""Autotuner table: keys by shape and step form, lookup order (user table
first, then the shipped one), and the plan config picks the entry up."""
import json

from spectral_galerkin_heat_b200 import autotune
from spectral_galerkin_heat_b200._lib import SghConfig


def _cfg(nx, ny, nz, latent=False):
    c = SghConfig()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.L_f = 2.7e5 if latent else 0.0
    return c


def test_keys_and_lookup(tmp_path, monkeypatch):
    assert autotune.key_of(_cfg(128, 64, 32)) == "128x64x32:face"
    assert autotune.key_of(_cfg(128, 64, 32, latent=True)) == "128x64x32:volume"
    table = tmp_path / "t.json"
    table.write_text(json.dumps({"entries": {"40x20x6:face": {"axis_min_ctas": 264}}}))
    monkeypatch.setenv("SGH_TUNE_TABLE", str(table))
    autotune._cache.clear()
    assert autotune.lookup(_cfg(40, 20, 6)) == 264
    assert autotune.lookup(_cfg(40, 20, 7)) is None  # in neither table: built-in default
    autotune._cache.clear()


def test_kernel_choice_and_box_form(tmp_path, monkeypatch):
    c = _cfg(80, 48, 120, latent=True)
    c.box = 1
    assert autotune.key_of(c) == "80x48x120:box"
    table = tmp_path / "t.json"
    table.write_text(json.dumps({"entries": {
        "80x48x120:box": {"axis_min_ctas": 132, "axis_cuda_cores": 1},
        "40x20x6:face": {"axis_min_ctas": 264}}}))
    monkeypatch.setenv("SGH_TUNE_TABLE", str(table))
    autotune._cache.clear()
    assert autotune.lookup_kernel(c) == 1
    assert autotune.lookup_kernel(_cfg(40, 20, 6)) is None   # entries without a kernel choice
    assert autotune.lookup_kernel(_cfg(41, 20, 6)) is None   # no entry
    autotune._cache.clear()


def test_batch_lookup_exact_then_same_classes(tmp_path, monkeypatch):
    """A batch mix is looked up by its exact key first; a batch that holds
    other slot counts of the same classes (a serving batch dealt over lanes)
    takes the entry of that class set; another class set finds nothing."""
    full = [_cfg(64, 32, 16)] * 4 + [_cfg(128, 64, 16)] * 4
    half = [_cfg(64, 32, 16)] * 2 + [_cfg(128, 64, 16)] * 2
    other = [_cfg(64, 32, 16)] * 2
    table = tmp_path / "t.json"
    table.write_text(json.dumps({"batch_entries": {
        autotune.batch_key(full, "mixed"): {"policy": {"vol_unroll": 8, "vol_vec": 2}}}}))
    monkeypatch.setenv("SGH_TUNE_TABLE", str(table))
    autotune._cache.clear()
    assert autotune.lookup_batch(full, "mixed") == {"vol_unroll": 8, "vol_vec": 2}
    assert autotune.lookup_batch(half, "mixed") == {"vol_unroll": 8, "vol_vec": 2}
    assert autotune.lookup_batch(other, "mixed") is None
    assert autotune.lookup_batch(half, "fp64") is None
    autotune._cache.clear()
