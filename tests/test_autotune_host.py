"""Host-side logic of the autotuner (no GPU): size classes, candidate
lists and the JSON cache."""
import json


def test_size_class_buckets():
    from dosecuda_b200 import autotune
    assert autotune.size_class(10485760, 15000, 4) == "V2^23_S2^14_B4"
    assert autotune.size_class(1, 1, 1) == "V2^0_S2^0_B1"


def test_variants_and_batch_candidates():
    from dosecuda_b200 import autotune
    names = autotune.variants()
    assert len(names) >= 2 and names[0] == "l8x8x8_c2"
    cands = autotune.batch_candidates()
    for v, bps in cands:
        assert 0 <= v < len(names)
        assert 2 <= bps <= autotune.max_blocks_per_sm(names[v])
    assert autotune.max_blocks_per_sm("t128_v4_c1") == 6
    assert autotune.max_blocks_per_sm("t128_v4_c2") == 5
    assert autotune.max_blocks_per_sm("t256_v2_c1") == 3
    assert (6, 6) in cands and names[6] == "t128_v4_c1"
    # the line family: voxel-tile shapes as well as round sizes are tuned
    lines = [n for n in names if autotune.shape_of(n)[0] == "l"]
    assert {autotune.shape_of(n)[1] for n in lines} >= {(8, 8, 8), (8, 8, 4), (8, 4, 8),
                                                        (8, 16, 8), (8, 8, 16)}
    assert autotune.shape_of("l8x8x4_c4") == ("l", (8, 8, 4), 32, 4)
    assert autotune.round_size("l8x8x8_c4") == 256 == autotune.round_size("t128_v4_c2")
    assert not autotune.same_decisions("l8x8x8_c4", "t128_v4_c2")
    assert autotune.same_decisions("t128_v4_c2", "t256_v2_c1")
    assert autotune.max_blocks_per_sm("l8x8x4_c4") == 20
    assert autotune.batch_shape("l8x4x8_c4") and not autotune.batch_shape("l8x8x16_c2")
    assert {names[v] for v, _ in cands} == {n for n in names if autotune.batch_shape(n)}
    # the default forward shape, and the batch's own default when the
    # persistent kernel cannot take it
    assert names[autotune.default_variant()] == "l8x16x8_c2"
    assert names[autotune.default_batch_variant()] == "l8x8x8_c2"


def test_cache_roundtrip(tmp_path, monkeypatch):
    from dosecuda_b200 import autotune
    path = tmp_path / "c" / "tune.json"
    monkeypatch.setenv("DOSECUDA_B200_TUNE_CACHE", str(path))
    assert autotune.cache_path() == str(path)
    autotune._store(str(path), "k1", [2, {"0": 1.5}])
    autotune._store(str(path), "k2", [0, 3])
    data = json.loads(path.read_text())
    assert data["k1"][0] == 2 and data["k2"] == [0, 3]
    assert autotune._load(str(tmp_path / "missing.json")) == {}
