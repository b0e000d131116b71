"""The launch-shape autotuner's host logic (umagnus_b200/autotune.py): the
candidate lists, the coordinate-descent search with a fake timer, and the
JSON cache.  The GPU side (every shape gives bit-identical results) is in
test_gpu_engine.py."""
import json

from umagnus_b200 import autotune as A


def test_torque_blocks_fit_the_kernel():
    for nx in (1, 5, 32, 64, 100, 256, 1024):
        blocks = A.torque_blocks(nx)
        assert blocks, nx
        for bx, by in blocks:
            assert bx % 32 == 0 and 64 <= bx * by <= 256
            assert bx <= max(32, (nx + 31) // 32 * 32)
    assert (32, 8) in A.torque_blocks(256) and (256, 1) in A.torque_blocks(256)
    assert all(bx == 32 for bx, _ in A.torque_blocks(5))


def test_search_finds_the_separable_minimum():
    # a fake timer whose optimum is torque 64x2 with global loads, stage 128/16, err 8
    def measure(kind, t):
        bx, by = t["torque_block"]
        c = abs(bx - 64) / 64 + abs(by - 2) / 2 + 0.1 * t["torque_tma"]
        c += abs(t["stage_threads"] - 128) / 128 + abs(t["stage_waves"] - 16) / 16 + abs(t["err_waves"] - 8) / 8
        return 1.0 + c

    best, log = A.search(measure, 256)
    assert best == {"torque_block": [64, 2], "stage_threads": 128, "stage_waves": 16, "err_waves": 8,
                    "torque_tma": 0}
    assert len(log["torque"]) == 2 * len(A.torque_blocks(256))
    assert len(log["stage"]) == len(A.STAGE_SHAPES) and len(log["err"]) == len(A.ERR_WAVES)
    assert A.DEFAULT["torque_block"] == [32, 8]  # the defaults are not modified


def test_cache_round_trip(tmp_path):
    path = tmp_path / "sub" / "tuning.json"
    assert A.load_cache(str(path)) == {}
    key = A.cache_key("NVIDIA B200", (256, 256, 16), "demag=1n|dmi=1|anis=1|regions=0")
    assert key == "NVIDIA B200|256x256x16|demag=1n|dmi=1|anis=1|regions=0"
    A.save_cache(str(path), {key: A.DEFAULT})
    assert A.load_cache(str(path)) == {key: A.DEFAULT}
    path.write_text("not json")
    assert A.load_cache(str(path)) == {}
    path.write_text(json.dumps([1, 2]))
    assert A.load_cache(str(path)) == {}
