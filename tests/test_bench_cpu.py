"""Host logic of bench.py that needs no GPU: the clock sampler keeps only the
nvidia-smi samples taken inside the timed region (or the nearest one when the
region is shorter than a sampling period), reads the throttle reasons from
the right columns, and reports an empty record as unsampled."""
import datetime
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _line(t, sm, reasons=("Not Active",) * 4):
    ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return ", ".join([ts, "0", str(sm), "1965", "700.00", "0x0"] + list(reasons)) + "\n"


def _sampler(lines):
    s = bench.ClockSampler(0)  # never started: stop() only parses its file
    s.out.write("".join(lines).encode())
    s.out.flush()
    return s


def test_samples_inside_the_timed_region_only():
    t0 = 1_800_000_000.0
    lines = [_line(t0 + 0.2 * k, 1000 + k) for k in range(20)]  # 4 s of samples
    lines[12] = _line(t0 + 2.4, 1500, ("Not Active", "Not Active", "Not Active", "Active"))
    clk = _sampler(lines).stop((t0 + 1.85, t0 + 2.65))
    # with the 0.1 s margin on each side: the samples at 1.8 .. 2.6 s
    assert clk["samples"] == 5
    assert clk["sampled"] == "timed region"
    assert clk["sm_mhz"] == 1011  # median of 1009, 1010, 1011, 1500, 1013
    assert clk["sm_max_mhz"] == 1965
    assert clk["reasons"] == ["sw_power_cap"]


def test_short_region_takes_the_nearest_sample():
    t0 = 1_800_000_000.0
    lines = [_line(t0 + 0.5 * k, 1200 + k) for k in range(10)]  # one sample every 0.5 s
    clk = _sampler(lines).stop((t0 + 1.2, t0 + 1.25))
    assert clk["samples"] == 1 and clk["sampled"] == "nearest sample to the timed region"
    assert clk["sm_mhz"] == 1202  # the sample at 1.0 s


def test_no_samples_is_unsampled():
    clk = _sampler([]).stop((0.0, 1.0))
    assert clk["reasons"] == ["unsampled"] and clk["sm_mhz"] is None


def test_tile_kernel_names_cover_every_shape_kind():
    # the library's tile table (read on the host, no GPU needed) names only
    # kernel kinds the bench can label
    import dnspir_b200 as dp
    kinds = {s[3] for s in dp.tscan_shapes()}
    assert kinds == set(range(len(bench.TILE_KERNELS)))
