"""Tile-shape choice of the grouped-GEMM autotuner (host logic, no GPU).

Every coupled-sector job takes the output-tile shape (0: 64x64, 1: 64x32,
2: 32x64, 3: 32x32) that minimises ntiles * (ceil(k/16) + 1) * cost[shape];
ties keep the lower shape index.
"""

import ctypes as C

import numpy as np
import pytest

from tenet_b200 import _lib

JOBS = [(80, 80, 100), (437, 437, 300), (20, 300, 50), (300, 20, 50)]


def cplan(jobs):
    rows, a, b, c = [], 0, 0, 0
    for m, n, k in jobs:
        rows.append([m, n, k, a, b, c, m, k, m])
        a, b, c = a + m * k, b + k * n, c + m * n
    arr = np.asarray(rows, dtype=np.int64)
    h = C.c_void_p()
    _lib.call("tnt_cplan_from_jobs", len(jobs), arr.ctypes.data_as(C.POINTER(C.c_int64)), a, b, c, C.byref(h))
    return h


def shapes(jobs, costs):
    h = cplan(jobs)
    try:
        out = np.zeros(len(jobs), dtype=np.int32)
        cs = np.asarray(costs, dtype=np.float64)
        _lib.call("tnt_cplan_tile_shapes", h, cs.ctypes.data_as(C.POINTER(C.c_double)),
                  out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out.tolist()
    finally:
        _lib.lib().tnt_cplan_destroy(h)


def test_equal_per_flop_costs_minimise_padding():
    assert shapes(JOBS, [1.0, 0.5, 0.5, 0.25]) == [3, 0, 2, 1]


def test_equal_per_tile_costs_keep_large_tiles():
    assert shapes(JOBS, [1.0, 1.0, 1.0, 1.0]) == [0, 0, 0, 0]


def test_expensive_small_tiles_only_for_thin_sectors():
    # a 20-row sector fits one 32-row tile as well as one 64-row tile
    assert shapes(JOBS, [1.0, 0.9, 0.9, 0.9]) == [0, 0, 2, 1]


@pytest.mark.parametrize("m,n", [(1, 1), (33, 65), (64, 64), (65, 31)])
def test_choice_is_a_minimum(m, n):
    costs = [1.0, 0.62, 0.58, 0.41]
    (s,) = shapes([(m, n, 40)], costs)
    dims = [(64, 64), (64, 32), (32, 64), (32, 32)]
    est = [-(-m // bm) * -(-n // bn) * costs[i] for i, (bm, bn) in enumerate(dims)]
    assert est[s] == min(est)
