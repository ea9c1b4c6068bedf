"""The reference arm of bench.py (the reference's own CPU direct sum on the host
cores) keeps the one-JSON-line contract, alone and under torchrun with two
ranks, where rank 0 alone measures and prints.  Runs on the CPU."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference library not built")


def _json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check_line(d):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "pair-interactions/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["config"]["workload"] == "two_stream_precision_form"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and "targets" in cb["sample"]
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--cpu-seconds", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0])


def test_reference_arm_under_two_ranks():
    env = dict(os.environ, MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", "29613", "bench.py", "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-seconds", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    _check_line(lines[0])
    assert lines[0]["n_gpus"] == 2


def test_reference_arm_loads_no_product_library():
    """The reference arm times the reference alone: the product's CUDA library
    is never mapped into its process."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
            "'--cpu-seconds', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_MAPPED' if 'libfs_b200' in maps else 'PRODUCT_NOT_MAPPED')")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_NOT_MAPPED" in r.stdout


def test_reference_arm_config_is_the_workload_config():
    """Both arms describe the workload with the same config dict."""
    sys.path.insert(0, ROOT)
    import bench
    from multi_species_b200 import decks
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--cpu-seconds", "1"], cwd=ROOT, capture_output=True, text=True, timeout=300)
    line = _json_lines(r.stdout)[0]
    d = decks.two_stream(h=8, ph=1, steps=100, remesh_period=5)
    assert line["config"] == bench.workload_config("two_stream_precision_form", d, decks.deck_points(d), 1)
