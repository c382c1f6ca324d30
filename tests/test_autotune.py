"""Host side of the autotuner: workload classes and the persisted tuning table.

The timing itself needs a GPU (tests/test_gpu_portfolio.py, tests/test_gpu_sort_join.py);
what is checked here is that tuned parameters are keyed by workload class and survive a
round trip through the JSON file, so a tuned process and a later one use the same shapes.
"""
import json
import math

from carmichael_frontier_b200 import autotune, workloads
from carmichael_frontier_b200.solve import Instance, Tuning


def _inst(w):
    return Instance.build(w.M, w.Q, w.B0, w.r, w.B)


def test_workload_class_is_radius_and_log_side_sizes():
    w = workloads.config1()
    inst = _inst(w)
    nD, nI = math.comb(len(inst.B0), 2), math.comb(len(inst.INS), 2)
    assert (nD, nI) == (406, 12246)                      # C(29, 2), C(157, 2)
    assert autotune.workload_class(inst) == f"r2_d{int(math.log2(nD))}_i{int(math.log2(nI))}"
    # the same modulus at another radius is another class
    a, b = workloads.config2(5), workloads.config2(5, r=4)
    assert autotune.workload_class(_inst(a)) != autotune.workload_class(_inst(b))


def test_tuning_cache_round_trips_through_its_file(tmp_path):
    path = str(tmp_path / "tuning.json")
    inst = _inst(workloads.config1())
    cache = autotune.TuningCache(path)
    assert cache.get(inst) is None
    tu = Tuning(d_per_part=3500, gen_shape=2, isplit=4, strategy="partition")
    cache.put(inst, tu)
    with open(path) as f:
        table = json.load(f)
    assert list(table) == [autotune.workload_class(inst)]
    again = autotune.TuningCache(path).get(inst)
    assert again == tu
    # a cached class is returned without timing anything (no GPU is touched here)
    assert autotune.TuningCache(path).tuned(inst) == tu
