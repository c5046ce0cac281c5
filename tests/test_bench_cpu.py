"""Host-side pieces of bench.py that need no GPU: the child-process ensemble record (its
result, failure and time-limit paths, with stand-in commands) and the host core count."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _py(code):
    return [sys.executable, "-c", code]


def test_ensemble_record_is_the_childs_last_json_line():
    rec = bench.ensemble_isolated(
        _py("import json; print('warming up'); print(json.dumps({'ensemble': {'batched_solves_per_s': 1.5}}))"), 60)
    assert rec == {"batched_solves_per_s": 1.5}


def test_failed_child_gives_unavailable_with_its_last_error_line():
    rec = bench.ensemble_isolated(_py("import sys; print('boom', file=sys.stderr); sys.exit(3)"), 60)
    assert "unavailable" in rec and "exited 3" in rec["unavailable"] and "boom" in rec["unavailable"]


def test_child_without_a_record_gives_unavailable():
    rec = bench.ensemble_isolated(_py("print('no json here')"), 60)
    assert rec == {"unavailable": "the ensemble run printed no record"}


def test_child_over_its_time_limit_is_stopped():
    rec = bench.ensemble_isolated(_py("import time; time.sleep(30)"), 1)
    assert rec == {"unavailable": "the ensemble run exceeded 1 s"}


def test_host_cores_within_the_affinity_mask():
    n = bench.host_cores()
    assert 1 <= n <= len(os.sched_getaffinity(0))
