"""CPU: bench.py's host-side choices. The encoder headline is the fastest
pruning policy within the 1% cost bound (the cheapest when none is), and
the CPU sample spreads its pictures over the whole batch (all QPs)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _p(speedup, cost):
    return {"speedup": speedup, "cost_increase_pct": cost}


def test_headline_is_the_fastest_policy_within_the_bound():
    pols = [_p(4.0, 3.0), _p(1.2, 0.9), _p(1.5, 1.0), _p(5.4, 7.2), _p(1.1, 0.4)]
    assert bench.pick_headline(pols) is pols[2]


def test_headline_without_a_policy_within_the_bound_is_the_cheapest():
    pols = [_p(4.0, 3.0), _p(2.0, 1.5), _p(5.4, 7.2)]
    assert bench.pick_headline(pols) is pols[1]


def test_cpu_sample_spreads_over_the_batch():
    idx = bench.sample_indices(128, 64)
    assert len(idx) == 64 and len(set(idx)) == 64
    assert {i // 32 for i in idx} == {0, 1, 2, 3}  # every QP group of 32 pictures
    assert bench.sample_indices(4, 16) == [0, 1, 2, 3]


def test_reference_arm_prints_the_contract_line():
    import json
    import subprocess

    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "Mpx/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["value"] > 0
    assert d["config"]["workload"] == bench.workload_name(32)
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"] == {"value": d["value"], "unit": "Mpx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_frame_sources_task_makes_the_workload_frame():
    """The generator pool's task returns frame f of the rank's content stream
    at the workload's coded size (what encoded_workload encodes)."""
    import numpy as np

    bench.load_pkg()
    from rustmpeg_next_b200 import synth

    got = bench._frame_sources(5, 1)
    _, _, p = synth.workload_picture(5, 32, bench.QPS)
    want = synth.workload_sources(5, p, 1)
    assert got[0].shape == (bench.CODED_H, bench.PIX_W)
    assert all(np.array_equal(a, b) for a, b in zip(got, want))


def test_general_section_tasks():
    """The coding-tree section's pool tasks: one synthetic picture, and its
    parity count (zero against the oracle's own planes, nonzero when one
    sample is off)."""
    import numpy as np
    import oracle

    oracle.build()
    part = bench._general_part(dict(vis_w=96, vis_h=64, ctu=32, bd=8, qp=30, seed=5))
    planes = [p.copy() for p in oracle.general_picture(*part)]
    assert bench._general_parity((part, planes)) == 0
    planes[1][3, 4] ^= 1
    assert bench._general_parity((part, planes)) == 1
    assert planes[0].shape == (64, 96) and planes[1].dtype == np.uint16
