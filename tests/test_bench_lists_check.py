"""The bench's whole-scene list check against the reference's viewshed stage
(bench.lists_vs_reference), with the reference stage stood in by a fake:
equal lists read "bit-exact", a planted difference names its voxel, and a
failing reference run is recorded rather than raised."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _lists():
    rng = np.random.default_rng(4)
    cnt = rng.integers(0, 6, 10)
    off = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    ids = rng.integers(1, 100, int(off[-1])).astype(np.int32)
    bcnt = cnt * 2 + 1
    boff = np.concatenate([[0], np.cumsum(bcnt)]).astype(np.int64)
    bb = rng.integers(0, 256, int(boff[-1])).astype(np.uint8)
    sh = rng.integers(0, 2 ** 31, (10, 3)).astype(np.uint32)
    return {"csr_off": off, "csr_ids": ids, "barle_off": boff, "barle": bb, "shadow": sh, "shadow_words": 3}


class FakeOracle:
    def __init__(self, ref=None, fail=False, built=True):
        self.ref, self.fail, self.built = ref, fail, built

    def ref_gpu(self):
        return object() if self.built else None

    def ref_stage1(self, scene):
        if self.fail:
            raise RuntimeError("ref_stage1 failed: 2")
        return self.ref

    @staticmethod
    def svf_to_words32(svf, words):
        return svf


class Scene:
    num_total = 10


def _ref_of(r):
    return {"csr_off": r["csr_off"].copy(), "csr_ids": r["csr_ids"].copy(), "barle_off": r["barle_off"].copy(),
            "barle": r["barle"].copy(), "svf": r["shadow"].copy()}


def test_equal_lists_are_bit_exact():
    r = _lists()
    res = bench.lists_vs_reference(FakeOracle(_ref_of(r)), Scene(), r)
    assert res["result"] == "bit-exact" and res["voxels"] == 10


def test_a_planted_difference_names_its_voxel():
    r = _lists()
    for key, voxel in (("csr_ids", None), ("barle", None), ("svf", 6)):
        ref = _ref_of(r)
        if key == "svf":
            ref["svf"][voxel, 1] ^= 4
        else:
            off = r["csr_off"] if key == "csr_ids" else r["barle_off"]
            voxel = int(np.flatnonzero(np.diff(off) > 0)[2])
            ref[key][off[voxel]] ^= 1
        res = bench.lists_vs_reference(FakeOracle(ref), Scene(), r)
        assert res["result"] == "DIFFERENT" and res["first_differing_voxel"] == voxel, key
    ref = _ref_of(r)
    ref["csr_off"][5:] += 1   # voxel 4 one id longer
    ref["csr_ids"] = np.concatenate([ref["csr_ids"], [7]]).astype(np.int32)
    res = bench.lists_vs_reference(FakeOracle(ref), Scene(), r)
    assert res["result"] == "DIFFERENT" and res["first_differing_voxel"] == 4


def test_a_failing_reference_run_is_recorded():
    r = _lists()
    assert bench.lists_vs_reference(FakeOracle(fail=True), Scene(), r)["result"] == "unavailable"
    res = bench.lists_vs_reference(FakeOracle(built=False), Scene(), r)
    assert res["result"] == "unavailable" and "not built" in res["why"]
