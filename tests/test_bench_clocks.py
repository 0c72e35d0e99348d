"""bench.py's clock record keeps only the nvidia-smi samples taken inside the
timed region (and says so), with throttle reasons from those samples only."""

import datetime
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _line(t, mhz, power_cap):
    ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    cap = "Active" if power_cap else "Not Active"
    return (f"{ts}, 0, {mhz}, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, {cap}\n")


def test_samples_outside_the_timed_region_are_dropped(tmp_path):
    import bench

    now = time.time()
    c = bench.ClockSampler(0)
    c.path = str(tmp_path / "clocks.csv")
    with open(c.path, "w") as f:
        f.write(_line(now - 1.0, 345, True))         # idle, before the region
        for k in range(5):
            f.write(_line(now + 0.02 * k, 1900 + k, False))
        f.write(_line(now + 2.0, 345, True))         # after the region
    c.mark(now - 0.001, now + 0.1)
    s = c.summary()
    assert s["samples"] == 5 and s["samples_from"] == "timed region"
    assert s["sm_mhz"] == 1902.0 and s["reasons"] == []


def test_short_region_falls_back_to_every_sample(tmp_path):
    import bench

    now = time.time()
    c = bench.ClockSampler(0)
    c.path = str(tmp_path / "clocks.csv")
    with open(c.path, "w") as f:
        f.write(_line(now, 1965, True))
    c.mark(now + 5.0, now + 5.01)
    s = c.summary()
    assert s["samples"] == 1 and s["reasons"] == ["sw_power_cap"]
    assert s["samples_from"].startswith("whole sampler run")
