"""CPU test of bench.py's clock sampler: it keeps the nvidia-smi samples whose own timestamps fall
in the timed region (not the time their lines were read) and reports the throttle reasons seen
there."""
import datetime
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _line(t, sm, reasons=("Not Active",) * 4):
    stamp = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return ", ".join([stamp, "0", str(sm), "1965", "700.0", "0x0", *reasons])


def test_samples_are_selected_by_their_own_timestamps():
    cs = bench.ClockSampler(0)
    cs.INTERVAL_MS = 1  # keep the test's sleep short
    cs.proc = _proc = _Proc()
    t0 = 1_800_000_000.0
    cs.t_mark = t0
    # read late and all at once (as a buffered pipe would deliver them): read times are useless
    late = t0 + 100.0
    cs.lines = [
        (late, _line(t0 - 5.0, 900, ("Not Active", "Active", "Not Active", "Not Active"))),  # before: ignored
        (late, _line(t0 + 0.01, 1965)),
        (late, _line(t0 + 0.03, 1950, ("Not Active", "Not Active", "Not Active", "Active"))),
        (late, "garbage line"),
    ]
    real_time = bench.time.time
    bench.time.time = lambda: t0 + 0.05  # end of the timed region
    try:
        out = cs.stop()
    finally:
        bench.time.time = real_time
    assert out["samples"] == 2
    assert out["sm_mhz"] == 1957.5 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]  # the hw_slowdown sample lies outside the region
    assert _proc is cs.proc
