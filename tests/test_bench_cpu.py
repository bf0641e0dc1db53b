"""bench.py's algorithmic work count, on CPU.

The roofline of the bench line divides the algorithmic FP32 work per pixel by
the fused kernel's time.  The count is the per-stage formula of the NL-SAR
path (similarities, box sums, weights, ENL statistics, selection, weighted
mean); these tests pin it to the worked figures of the headline settings and
check that it follows the patch and scale sets.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_headline_counts():
    # patches {3,5,7}, scales {1,3}, search 21
    assert bench.flop_per_pixel("argmax_enl") == 57956
    # reference selection computes only the last statistics key
    assert bench.flop_per_pixel("reference") == 15066


def test_count_follows_the_combinations():
    base = bench.flop_per_pixel("argmax_enl", [3], [1])
    # each extra (patch, scale) combination adds the same per-combination work
    per_combo = bench.flop_per_pixel("argmax_enl", [3, 5], [1]) - base
    assert bench.flop_per_pixel("argmax_enl", [3, 5, 7], [1]) - base == 2 * per_combo
    # the reference example's settings: 15 combinations over 3 scales
    assert bench.flop_per_pixel("argmax_enl", [3, 5, 7, 9, 11], [1, 3, 5]) == 132694
    # reference selection does not depend on how many keys exist
    assert bench.flop_per_pixel("reference", [3, 5, 7, 9, 11], [1, 3, 5]) == 15066
