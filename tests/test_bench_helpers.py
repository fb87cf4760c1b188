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


class _DoneProcess:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _sampler_with(lines, window):
    s = bench.ClockSampler(0)
    s.proc = _DoneProcess()
    s._t = SimpleNamespace(join=lambda timeout=None: None)
    s.lines = lines
    s.window = window
    return s


def test_clock_samples_are_kept_inside_the_timed_region():
    # index, clocks.sm, clocks.max.sm, power, active, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    idle = "0, 1200, 1965, 150, 0x0, Not Active, Not Active, Not Active, Not Active"
    busy = "0, 1965, 1965, 900, 0x4, Not Active, Not Active, Not Active, Active"
    lines = [(0.0, idle), (1.0, busy), (1.1, busy), (1.2, busy), (3.0, idle)]
    got = _sampler_with(lines, (0.9, 1.25)).stop()
    assert got["samples"] == 3 and got["in_timed_region"]
    assert got["sm_mhz"] == 1965.0 and got["sm_max_mhz"] == 1965.0
    assert got["reasons"] == ["sw_power_cap"]


def test_clock_samples_fall_back_to_all_when_none_is_inside():
    idle = "0, 1200, 1965, 150, 0x0, Not Active, Not Active, Active, Not Active"
    got = _sampler_with([(0.0, idle), (0.5, idle)], (2.0, 2.1)).stop()
    assert got["samples"] == 2 and not got["in_timed_region"]
    assert got["reasons"] == ["sw_thermal_slowdown"]
