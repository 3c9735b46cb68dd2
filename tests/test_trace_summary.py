"""The bench's summary of a level kernel's pass timeline (bench.trace_summary)
on a hand-made timeline: two instances, one waiting CTA, one ordered walk."""
import importlib.util
import os

import numpy as np
from pytest import approx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_for_trace", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def test_trace_summary_of_a_small_timeline():
    b = _bench()
    # (t ns, event, value): instance 0 runs a trial pass then finishes;
    # instance 1 runs a gradient pass, a summary pass, then finishes
    ev = [
        (0, 1, (0 << 8) | 6), (100, 1, (1 << 8) | 1),
        (1000, 2, (0 << 8) | 6), (1200, 1, (0 << 8) | 13),
        (2000, 2, (1 << 8) | 1), (2100, 1, (1 << 8) | 12),
        (3000, 2, (1 << 8) | 12), (3100, 4, 500), (3700, 1, (1 << 8) | 13),
        (1300, 3, 2000),   # a CTA waits 2 us after instance 0 finished
        (50, 3, 600),      # and one waits 0.6 us before
    ]
    ev.sort()
    tr = {"t": np.array([e[0] for e in ev], dtype=np.int64),
          "event": np.array([e[1] for e in ev], dtype=np.int32),
          "cta": np.zeros(len(ev), dtype=np.int32),
          "value": np.array([e[2] for e in ev], dtype=np.int64)}
    s = b.trace_summary(tr, ctas=2)
    assert s["span_ms"] == approx(3700 / 1e6)
    assert s["idle_cta_ms"] == approx(2600 / 1e6)
    assert s["idle_cta_ms_after_first_finish"] == approx(2000 / 1e6)
    assert s["finish_ms"] == approx([1200 / 1e6, (1200 + 3700) / 2 / 1e6, 3700 / 1e6])
    assert s["walks"] == 1 and s["walk_us_mean"] == approx(0.5)
    assert s["pass_us"]["trial"] == [1, approx(1.0)]
    assert s["pass_us"]["gradient"] == [1, approx(1.9)]
    assert s["pass_us"]["xsum"] == [1, approx(0.9)]
    # control step: from a completion to the instance's next publication
    assert s["control_us"]["gradient"] == approx(0.1)
    assert s["control_us"]["trial"] == approx(0.2)
    assert s["control_us"]["xsum"] == approx(0.7)
