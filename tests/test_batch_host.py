"""Host logic of the batched driver that needs no GPU: which instances the
autotuner times for a shape."""
from canary_b200 import batch as B


def test_tuning_picks_follow_the_workload_then_repeat_it():
    inst = [(2, 4, 6), (2, 5, 9), (2, 4, 10), (3, 4, 4), (2, 4, 8)]
    # 2-D N=4: 25 nodes per element; the workload's own three instances hold 5000 nodes
    picks, distinct, nodes = B.tuning_picks(inst, 2, 4, 12000)
    assert distinct == 3
    assert picks[:3] == [6, 10, 8]
    assert picks[3:] == [6, 10, 8, 6, 10][:len(picks) - 3]  # repeated in the same order
    assert nodes == sum(ns * ns * 25 for ns in picks) and nodes >= 12000
    assert nodes - picks[-1] ** 2 * 25 < 12000  # stops as soon as the target is reached


def test_tuning_picks_stop_at_the_target_within_the_workload():
    inst = [(3, 7, 16), (3, 7, 16), (3, 7, 16)]
    picks, distinct, nodes = B.tuning_picks(inst, 3, 7, 16 ** 3 * 512 + 1)
    assert picks == [16, 16] and distinct == 2 and nodes == 2 * 16 ** 3 * 512


def test_tuning_picks_of_an_absent_shape_are_empty():
    assert B.tuning_picks([(2, 4, 6)], 2, 5, 1000) == ([], 0, 0)
