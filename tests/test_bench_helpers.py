"""Host-side helpers of bench.py (no GPU needed): the solve-time-to-M_dot metric, the roofline arithmetic and the
adjoint case."""
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


def _run(precision="fp64", inner=4, passes=2, steps=2):
    return {"n_cells": 1000, "nv": 512, "inner": inner, "passes": passes, "device_s": 0.42 * steps,
            "timings": {"gradient": 0.1 * steps, "residual": 0.12 * steps, "sweep_forward": 0.2 * steps,
                        "sweep_backward": 0.0}, "lout_bytes_per_unit": None}


def test_step_fraction_counts_the_path_bytes_per_unit():
    """Per CIS iteration and (cell, velocity): inner x (3 s_F + 2 s_W + 3 s_W per further block pass) + s_F for the
    moments: 264 B in FP64 and 132 B in FP32 storage at 4 inner sweeps and 2 block passes."""
    r = bench.step_fraction(_run(), "fp64", 2, 6000.0)
    assert r["bytes_per_unit_per_iteration"] == 264
    assert abs(r["achieved"] - 264 * 1000 * 512 / 0.42 / 1e9) < 1e-12
    assert abs(r["frac"] - r["achieved"] / 6000.0) < 1e-15
    assert bench.step_fraction(_run(), "mixed", 2, 6000.0)["bytes_per_unit_per_iteration"] == 132
    # the issue-rate bound: the sweeps at the full issue rate plus the other phases as measured (none here)
    ib = r["issue_bound"]
    rate = 148 * 128 * bench.sm_max_mhz() * 1e6
    t_min = 4 * sum(bench.INSTR_PER_UNIT["fp64"]) * 1000 * 512 / rate
    assert abs(ib["min_seconds_per_iteration"] - t_min) <= 1e-12 * t_min
    assert abs(ib["max_frac"] - 264 * 1000 * 512 / t_min / 1e9 / 6000.0) <= 1e-9 * ib["max_frac"]


def test_kernel_rooflines_divide_algorithmic_bytes_by_the_launch_time():
    import os

    os.environ.pop("KIN_SWEEP_KERNEL", None)
    os.environ.pop("KIN_MIXED_RESIDUAL", None)
    k = bench.kernel_rooflines(_run(), "fp64", 2, 6000.0)
    units = 1000 * 512
    g = k["k_gradient"]
    assert g["launches_per_step"] == 4 and g["bytes_per_unit"] == 32
    assert abs(g["achieved_gbs"] - 32 * units / (0.1 / 4) / 1e9) < 1e-9
    assert k["k_residual"]["bytes_per_unit"] == 40
    # two block passes: (2 s + 4 s) / 2 per launch, 8 launches per step
    t = k["k_sweep_tiles"]
    assert t["bytes_per_unit"] == 24 and t["launches_per_step"] == 8
    assert "k_lout" not in k
    assert bench.sweep_kernel_bytes(8, 1)[1] == 24 and bench.sweep_kernel_bytes(4, 3)[1] == (8 + 12 + 16) / 3


def test_adjoint_channel_uses_the_reference_default_scheme():
    setup, host = bench.channel_case(nv=6, n=(4, 2, 1))
    assert int(setup["discrete_eq"]) == 1 and host.pressure_boundary_reconstruction == "limited"
    setup, host = bench.channel_case(nv=6, n=(4, 2, 1), scheme="continuous-cell")
    assert int(setup["discrete_eq"]) == 0 and host.pressure_boundary_reconstruction == "cell"
