"""bench.py's reference arm on CPU: one JSON line with the contract's keys, at
least 3 warm-up steps, and under torchrun with two ranks only rank 0 works and
prints while the other exits 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["bench.py", "--impl", "reference", "--config", "c1", "--steps", "1", "--warmup", "0"]


def _env():
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        e.pop(k, None)
    e["OMP_NUM_THREADS"] = "2"
    return e


def _json_lines(out):
    return [json.loads(ln) for ln in out.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    r = subprocess.run([sys.executable] + ARGS, cwd=ROOT, capture_output=True, text=True, timeout=600, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    ln = lines[0]
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in ln, k
    assert ln["impl"] == "reference" and ln["n_gpus"] == 1 and ln["steps"] == 1 and ln["warmup"] >= 3
    assert ln["value"] > 0 and ln["higher_is_better"] is True and ln["unit"] == "timeslices/s"
    assert "workload" in ln["config"] and ln["data"] == "synthetic"
    cb = ln["cpu_baseline"]
    assert cb["value"] == ln["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    e = ln["e2e"]
    assert e["value"] == ln["value"] and e["unit"] == ln["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert abs(ln["ms_per_step"] - 1000.0 / ln["value"]) <= 1e-6 * ln["ms_per_step"]


def test_reference_arm_two_ranks_rank0_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", "29517"] + ARGS + ["--gpus", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


def test_lime_io_measurement_small():
    sys.path.insert(0, ROOT)
    import bench
    out = bench.measure_lime_io(L=4, T=3)
    assert out["matches_written"] and out["oracle_matches"]
    assert out["bytes"] == 4 ** 3 * 3 * 72 * 8 and out["cold_gbs"] > 0 and out["warm_gbs"] > 0
    assert not [p for p in os.listdir(ROOT) if p.startswith("_lime_")]


def test_reference_arm_per_core_layout():
    """The reference's MPI layout (one single-threaded timeslice per core): same line, per-core throughput."""
    r = subprocess.run([sys.executable] + ARGS + ["--cpu-layout", "per-core"], cwd=ROOT, capture_output=True,
                       text=True, timeout=900, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1
    ln = lines[0]
    cb = ln["cpu_baseline"]
    assert ln["impl"] == "reference" and ln["value"] > 0 and cb["layout"] == "one timeslice per core"
    assert cb["cores"] == (os.cpu_count() or 1)
    assert abs(ln["ms_per_step"] * ln["value"] / 1000.0 - cb["cores"]) < 1e-6 * cb["cores"]


def test_reference_arm_never_loads_the_product_library():
    """The reference arm times the oracle's restatement of the reference path: its process must not import the
    product package nor map liblaph_gpu.so (its inputs come from the oracle's own field generator)."""
    code = ("import runpy, sys\n"
            "sys.argv = " + repr(ARGS + ["--no-per-core"]) + "\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit as e:\n    assert not e.code\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'liblaph_gpu' not in maps, 'liblaph_gpu.so mapped'\n"
            "assert not any(m.startswith('laph_eigsys_b200') for m in sys.modules), 'package imported'\n"
            "print('CLEAN')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600, env=_env())
    assert r.returncode == 0, r.stderr[-2000:]
    assert "CLEAN" in r.stdout
    line = _json_lines(r.stdout)[0]
    assert "inputs" in line["cpu_baseline"]
