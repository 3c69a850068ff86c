"""bench.py's output contract, checked on the CPU: the reference arm (the
single-precision CPU port of the reference's path on a bounded sample) prints
one JSON line with the keys the benchmark driver reads, for the same
workload, metric and unit as this library's arm; the algorithmic FLOP counts
behind the roofline are the FFTW-convention figures the design states."""
import json
import os
import subprocess
import sys

import bench
from mset_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_flop_counts_per_unit_and_position():
    # 4 FFTs of 128 x 128 (5 N^2 log2 N^2 each) + 32 N^2 pointwise per unit;
    # 6 FFTs + 40 N^2 per position
    assert bench.flops_per_unit(128) == 4 * 5 * 128 ** 2 * 14 + 32 * 128 ** 2 == 5111808
    assert bench.flops_per_position(128) == 6 * 5 * 128 ** 2 * 14 + 40 * 128 ** 2 == 7536640
    assert abs(bench.flops_per_unit(256) - 23.07e6) < 0.01e6


def test_reference_arm_prints_the_contract_line():
    env = dict(os.environ, OMP_NUM_THREADS="4")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, cwd=ROOT, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["metric"] == "slice-propagations/s (fwd+adjoint)" and d["unit"] == "slice-propagations/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    cfg = synth.CONFIGS["mid"]
    ns = -(-cfg.vol[0] // cfg.slice_binning)
    positions = cfg.scan[0] * cfg.scan[1] * cfg.n_tilts
    assert d["config"]["workload"] == bench.workload_name(cfg, ns, positions)
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
