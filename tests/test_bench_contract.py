"""bench.py's contract pieces that need no GPU: the reference arm's JSON line (the CPU
restatement timed on the host), the defaults, the schedule report and the committed
profile figures it reads."""
import json
import os
import subprocess
import sys

import pytest

import bench
from mdwtracker_b200 import MDWT_HOST_ONLY, Renderer

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=e,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_prints_the_contract_line():
    lines = run_bench(["--impl", "reference", "--config", "c1", "--steps", "1", "--warmup", "1"])
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["metric"] == "Gpath-samples/s" and line["unit"] == "Gpath-samples/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["scaling"] == "strong"
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 1 and line["vs_baseline"] is None
    assert line["config"]["workload"].startswith("c1_")
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "Gpath-samples/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    assert run_bench(["--impl", "reference", "--config", "c1"], env={"RANK": "1"}) == []


def test_defaults(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse_args()
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1 and a.config == "c3" and a.edge == 16 and a.impl == "mdwt"
    assert not a.no_autotune and a.regroup is None and a.split == "rows"
    # the headline line runs the exact arithmetic; the fast one is an extra key
    assert a.arith == "exact" and not a.no_fast


def test_headline_traffic_is_the_committed_full_frame_capture():
    t = bench.profiled_traffic("trace_regroup_kernel", "c3_syncdda_6x512f32_e16_mc32_1920x1080_256spp")
    assert t is not None and 1e9 < t < 1e10


def test_schedule_report_reads_the_knobs():
    r = Renderer(MDWT_HOST_ONLY)
    # a host-only context has no method yet (-m 0): the warp-local tracker by default
    assert bench.schedule_of(r, "default") == {"regroup": 0, "rg_blocks": 0, "trips": 4, "pool": 8, "quorum": 16,
                                               "by": "default"}
    r.setTuning(4, 0)
    r.setTuning(2, 6)
    s = bench.schedule_of(r, "x")
    assert s["regroup"] == 0 and s["trips"] == 6


@pytest.mark.parametrize("kernel,bytes_", [("trace_regroup_kernel", 94480640.0), ("trace_kernel", 92951552.0)])
def test_profiled_traffic_reads_the_committed_summaries(kernel, bytes_):
    assert bench.profiled_traffic(kernel, "c2_syncdda_3x256u8_mc16_1024x1024_64spp") == bytes_
    assert bench.profiled_traffic(kernel, "no_such_workload") is None
