"""The bench's reference arm (CPU only): one JSON line with the contract's
keys, the reference's serial step on every host core, and nothing from the
ranks other than 0."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "1"], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=900)


def test_reference_arm_line():
    p = _run({"RANK": "0"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and p.stdout.strip() == lines[0]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    cores = len(os.sched_getaffinity(0))
    assert d["cpu_baseline"]["cores"] == max(1, min(cores, 64))
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert "the whole grid" in d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1"})
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_reference_slab_plan():
    sys.path.insert(0, ROOT)
    import bench
    # the driver's 20 + 5 steps: the whole grid, one slab per core
    assert bench.ref_slab_plan(25, 16) == (16, 64)
    assert bench.ref_slab_plan(25, 8) == (8, 128)
    assert bench.ref_slab_plan(25, 1) == (1, 1024)
    # long runs: thinner slabs, a sample of the grid (multiples of 16 rows)
    procs, nz = bench.ref_slab_plan(2010, 16)
    assert procs == 16 and nz == 16 and procs * nz < bench.NZ
    assert bench.ref_slab_plan(100, 4) == (4, 256)         # the per-core share binds
    assert bench.ref_slab_plan(100, 1) == (1, 400)         # the time budget binds
    # never more processes than 16-row slabs
    assert bench.ref_slab_plan(25, 200)[0] == bench.NZ // 16
