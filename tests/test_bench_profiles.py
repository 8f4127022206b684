"""The bench line's roofline object reads per-launch figures of its dominant
kernel from the committed ncu summaries (profiles/<kernel>_1M_1080p.md):
DRAM traffic, executed warp instructions and instructions per blended pair.
Both compositing kernels' summaries must carry all three, with values that
agree with each other (instructions per pair = instructions / blended pairs
of the bench scene, 58,368,764 by the CPU oracle)."""
import pytest

import bench

BLENDED_PAIRS = 58_368_764  # bench/count_pairs.py on the bench scene and camera


@pytest.mark.parametrize("tag", ["k_draw_1M_1080p", "k_draw_backward_1M_1080p"])
def test_profiles_carry_the_roofline_figures(tag):
    traffic = bench.profile_figure(tag, "traffic_bytes_per_launch")
    inst = bench.profile_figure(tag, "warp_inst_per_launch")
    per_pair = bench.profile_figure(tag, "inst_per_blended_pair")
    assert traffic is not None and 1e7 < traffic < 1e9
    assert inst is not None and inst > 1e8
    assert per_pair is not None
    assert abs(per_pair - inst / BLENDED_PAIRS) < 0.01


def test_missing_profile_or_key_reads_as_none():
    assert bench.profile_figure("no_such_kernel", "traffic_bytes_per_launch") is None
    assert bench.profile_figure("k_draw_1M_1080p", "no_such_key") is None
