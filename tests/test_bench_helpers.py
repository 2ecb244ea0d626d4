"""bench.py's host-side pieces, without a GPU: the workload description, the
roofline figures it reads from committed files, the replica set it times,
and its argument checks."""

import importlib
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    return importlib.import_module("bench")


def test_config_names_the_workload(bench):
    c = bench.config(256000, 1)
    assert c["workload"] == "lj-fcc40x4-256k-rho0.8442-shifted-force-langevin-grid-on-list-trigger"
    assert c["particles_per_box"] == 256000 and c["parallelism"] == "replicas x1"
    assert "flushed" in c["l2"] and "grid" in c
    json.dumps(c)


def test_algorithmic_flops(bench):
    # 11 per list candidate, 26 per force-shifted pair: 77.6 and 55.25 at rho 0.8442
    f = bench.flops_per_particle_step(0.8442)
    assert abs(f - (11 * 77.62 + 26 * 55.25)) < 5.0


def test_roofline_inputs_from_committed_files(bench):
    peak, kind = bench.measured_peaks()
    assert peak > 1000.0 and kind in ("measured", "fallback")
    traffic = bench.profile_traffic()
    # the step kernel's DRAM bytes per launch from its committed ncu summary:
    # well above the 96 B x 256,000 algorithmic bytes (the list streams)
    assert traffic is not None and 96 * 256000 < traffic < 1e9


def test_roofline_picks_the_binding_roof(bench):
    # rho 0.8442: 2,290 flop against 96 B per particle-step, above the machine
    # balance, so the FP32 roof binds and its fraction is the headline
    line = bench.roofline_line(500.0, 6500.0, "measured", 11.5, 71.0, 2290.0, 1e8, 51e-6, 200)
    assert line["bound"] == "fp32" and line["unit"] == "TFLOP/s"
    assert abs(line["frac"] - 11.5 / 71.0) < 1e-12
    assert line["hbm"]["frac"] < line["frac"]
    line = bench.roofline_line(3000.0, 6500.0, "measured", 1.0, 71.0, 20.0, 1e8, 51e-6, 200)
    assert line["bound"] == "hbm" and line["unit"] == "GB/s"
    json.dumps(line)


def test_metric_and_unit(bench):
    assert bench.UNIT == "particle-steps/s"
    assert "batched vs plain" in bench.METRIC and bench.ALGO_BYTES == 96


def test_uneven_replica_set(vl):
    # the batched workload: N log-uniform in [500, 20000], rho in [0.01, 0.90]
    reps = vl.uneven_replicas(512, 2024)
    sizes = [len(r.particles) for r in reps]
    assert len(reps) == 512 and sum(sizes) == 2_786_089
    assert 500 <= min(sizes) and max(sizes) <= 20000
    densities = [len(r.particles) / (r.box_size[0] * r.box_size[1] * r.box_size[2]) for r in reps]
    assert 0.009 < min(densities) and max(densities) < 0.91


def test_warmup_below_three_is_refused(bench, monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--warmup", "2"])
    with pytest.raises(SystemExit) as e:
        bench.main()
    assert e.value.code == 2
