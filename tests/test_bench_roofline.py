"""The bench's roofline object (host arithmetic only): the dominant kernel is
the one with the most time per step, achieved = algorithmic work / time, and
the DRAM traffic of the update-matrix GEMM is the ncu-measured traffic per
algorithmic byte scaled to the launch size."""
import bench


def test_tensor_roofline_with_traffic():
    kern = {"gemm_u": {"ms_per_step": 25.0, "launches_per_step": 18, "gflop_per_step": 3300.0, "gb_per_step": 26.0},
            "build": {"ms_per_step": 8.7, "launches_per_step": 19, "gflop_per_step": 0.0, "gb_per_step": 27.0}}
    r = bench.roofline(kern, 240.0, "test", 6540.0, bench.TRAFFIC_PER_ALG_BYTE)
    assert r["kernel"] == "gemm_u" and r["bound"] == "tensor"
    assert abs(r["achieved"] - 132.0) < 1e-9 and abs(r["frac"] - 132.0 / 240.0) < 1e-12
    per_launch = 26.0 / 18 * 1e9
    ratio = bench.TRAFFIC_PER_ALG_BYTE["gemm_u"][0]
    assert abs(r["traffic"] - ratio * per_launch) < 1.0 and "traffic_source" in r


def test_hbm_roofline_without_capture():
    kern = {"build": {"ms_per_step": 8.7, "launches_per_step": 19, "gflop_per_step": 0.0, "gb_per_step": 27.2}}
    r = bench.roofline(kern, 240.0, "test", 6540.0)
    assert r["bound"] == "hbm" and r["traffic"] is None
    assert abs(r["achieved"] - 27.2 / 8.7 * 1e3) < 1e-6


def test_no_traffic_without_a_matching_capture():
    """FP64 and batch runs have no capture of their own: traffic stays null."""
    kern = {"gemm_u": {"ms_per_step": 25.0, "launches_per_step": 18, "gflop_per_step": 3300.0, "gb_per_step": 26.0}}
    r = bench.roofline(kern, 35.0, "test", 6540.0)
    assert r["traffic"] is None and "traffic_source" not in r
