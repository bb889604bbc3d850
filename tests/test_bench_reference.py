"""The reference arm of bench.py (the host-core CPU step, no GPU): its one JSON line carries the
keys the benchmark contract names, and ranks other than 0 of a multi-process launch exit quietly."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--atoms", "20000",
                           "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, env=env,
                          cwd=ROOT)


def test_reference_arm_line():
    res = run_bench({})
    assert res.returncode == 0, res.stderr
    lines = [x for x in res.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "atom-steps/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] >= 3
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    assert d["config"]["workload"] and d["config"]["atoms_per_gpu"] == 20000


def test_reference_arm_prints_the_same_config_as_the_gpu_arm():
    sys.path.insert(0, ROOT)
    import bench
    res = run_bench({})
    d = json.loads([x for x in res.stdout.splitlines() if x.startswith("{")][0])

    class A:
        atoms = 20000
    assert d["config"] == bench.config_of(A, 1)


def test_reference_arm_never_maps_the_engine_library():
    # the reference arm runs the CPU restatement only: the engine's shared library must not be loaded
    code = ("import sys, bench; sys.argv = ['bench.py', '--impl', 'reference', '--atoms', '5000', '--steps', '1', "
            "'--warmup', '0']; bench.main(); maps = open('/proc/self/maps').read(); "
            "print('ENGINE_MAPPED' if 'libdsmc_b200' in maps else 'ENGINE_NOT_MAPPED')")
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert res.returncode == 0, res.stderr
    assert "ENGINE_NOT_MAPPED" in res.stdout


def test_reference_arm_other_ranks_print_nothing():
    res = run_bench({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert res.returncode == 0, res.stderr
    assert not [x for x in res.stdout.splitlines() if x.startswith("{")]
