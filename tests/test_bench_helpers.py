"""Host-side helpers of bench.py that turn measurements into the reported
figures: launches per apply (the `gpu_launches` claim) against the committed
launch list, and the translation's FP64 flop count against the algorithmic
count of the 245,760-unknown workload."""
import sys
from pathlib import Path
from types import SimpleNamespace

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_launches_per_apply_matches_the_launch_list():
    # profiles/launches_fp64_apply_sphere_245760.md: one apply is 23 launches
    # at maxLevel 6 with the default kernels
    tune = {"m2l.variant": 4, "up.variant": 0, "l2l.variant": 1, "agg.variant": 0, "leaf.variant": 0}
    assert bench.launches_per_apply(6, tune) == 23
    assert bench.launches_per_apply(6, {**tune, "m2l.variant": 0}) == 29   # one translation per level
    assert bench.launches_per_apply(6, {**tune, "leaf.variant": 1}) == 24  # near field on its own
    assert bench.launches_per_apply(6, {**tune, "agg.variant": 1}) == 22   # both media in one aggregation


def test_translation_flops_of_the_full_workload():
    # interaction pairs and directions per level (2..6) of the 245,760-unknown sphere
    pairs = [576, 5408, 16464, 84648, 308808]
    k1 = [8450, 3042, 1250, 512, 288]
    k2 = [17672, 5832, 2178, 882, 450]
    op = SimpleNamespace(max_level=6, info=SimpleNamespace(far_pairs=pairs, K_k1=k1, K_k2=k2))
    assert bench.translation_flops(op) == 22338003456.0
