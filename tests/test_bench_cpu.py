"""Host-side helpers of bench.py (no GPU): the sysfs cpulist parser behind the NUMA placement
of the end-to-end staging buffers, and the whole-job throughput formula."""
import bench


def test_parse_cpulist():
    assert bench.parse_cpulist("0-3,8,10-11\n") == {0, 1, 2, 3, 8, 10, 11}
    assert bench.parse_cpulist("5") == {5}
    assert bench.parse_cpulist("") == set()


def test_whole_job_value_is_weak_scaling_total():
    # 2 ranks × 10 steps × 1 GFLOP in 20 ms (slowest rank) = 1000 GFLOP/s
    assert abs(bench.whole_job_value(1e9, 2, 10, 20.0) - 1000.0) < 1e-9
