"""Host logic of the learned warm-start evaluation (no GPU): hit times
against a reference objective and the per-start summary."""
import pytest

from yoricktrtt_b200.recon import VMLMBInfo
from yoricktrtt_b200.warmstart import TOLS, _hit, summarize


def test_hit_iteration_and_time():
    info = VMLMBInfo(iterations=4, f=[100.0, 10.0, 1.001, 1.00001, 1.0], times=[0.0, 0.1, 0.2, 0.3, 0.4])
    assert _hit(info, 1.0, 1e-2) == (2, 0.2)
    assert _hit(info, 1.0, 1e-4) == (3, 0.3)
    assert _hit(info, 1.0, 1e-6) == (4, 0.4)
    assert _hit(info, 0.5, 1e-6) == (None, None)


def _row(seed, f_ref, **starts):
    r = {"seed": seed, "f_ref": f_ref}
    for name, (it, sec, f, hit) in starts.items():
        d = {"seconds": sec, "start_seconds": 0.0, "iterations": it, "evaluations": it + 1, "f": f,
             "f_start": 10 * f, "converged": True, "rel_diff_vs_zero": 0.0}
        for tol in TOLS:
            d[f"to_{tol:g}"] = hit
        r[name] = d
    return r


def test_summary_speedups():
    rows = [_row(1, 1.0, zero=(100, 2.0, 1.0, {"iterations": 90, "seconds": 1.8}),
                 learned=(50, 1.0, 1.0, {"iterations": 45, "seconds": 0.9})),
            _row(2, 1.0, zero=(120, 2.4, 1.0, {"iterations": 110, "seconds": 2.2}),
                 learned=(60, 1.2, 1.0, None))]
    s = summarize(rows)
    assert s["zero"]["stop_rule"]["iterations_mean"] == 110
    assert s["learned"]["stop_rule"]["seconds_mean"] == pytest.approx(1.1)
    assert s["learned"]["speedup_vs_zero"]["stop_rule_seconds_mean"] == pytest.approx(2.2 / 1.1)
    assert s["learned"]["to_0.0001"]["reached"] == 1
    assert s["learned"]["speedup_vs_zero"]["to_0.0001_iterations_median"] == pytest.approx(100 / 45)
