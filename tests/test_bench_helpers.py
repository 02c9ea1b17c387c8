"""Host-side helpers of bench.py's solve-time-to-M_dot metric (no GPU needed)."""
import bench


def test_settle_time_is_the_first_time_after_which_mdot_stays_within_tolerance():
    ref = 1.0
    hist = [(1.0, 1.5, 0.0), (2.0, 1.00005, 0.0), (3.0, 1.001, 0.0), (4.0, 1.00002, 0.0), (5.0, 0.99999, 0.0)]
    assert bench.settle_time(hist, ref, 1e-4) == 4.0
    assert bench.settle_time(hist, ref, 1e-2) == 2.0
    assert bench.settle_time(hist, ref, 1e-6) is None


def test_settle_time_empty_and_never():
    assert bench.settle_time([], 1.0, 1e-4) is None
    assert bench.settle_time([(1.0, 2.0, 0.0)], 1.0, 1e-4) is None
