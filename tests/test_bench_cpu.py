"""bench.py's host logic on CPU: the self-launch of `--gpus N`, the rank
plumbing under gloo, the reference arm's sample and its isolation from this
package (it must time the reference's build alone, with none of this
library loaded into its process)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out):
    for line in reversed(out.strip().splitlines()):
        line = line.strip()
        if line.startswith("{"):
            return json.loads(line)
    raise AssertionError("no JSON line in:\n" + out)


def test_gpus_2_launches_two_ranks():
    env = dict(os.environ, OMP_NUM_THREADS="1")
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--plumbing",
                        "--steps", "3", "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    j = _last_json(r.stdout)
    assert j["n_gpus"] == 2
    assert j["plumbing"]["ranks_reporting"] == 2
    # weak scaling: each rank its own 64-disk draw, and the config counts both
    assert j["config"]["disks"] == 128
    assert j["plumbing"]["cells"] == j["config"]["cells"]


def test_reference_arm_loads_nothing_of_the_package():
    code = (
        "import sys, bench\n"
        "class A: workload='c4'; strong=False; groups=4\n"
        "cfg = bench.workload_config(A, 1)\n"
        "s = bench.reference_sample(bench.workload_disks('c4'), 20, 5)\n"
        "assert not any(m.startswith('cudaprotoplanetarydisksfloat_b200') for m in sys.modules), sorted(sys.modules)\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libfargo_b200' not in maps\n"
        "print(cfg['disks'], len(s))\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split() == ["64", "5"]


@pytest.mark.parametrize("K,W", [(20, 5), (3, 3), (100, 5), (7, 10)])
def test_reference_sample_shares(K, W):
    sys.path.insert(0, ROOT)
    import bench
    disks = bench.workload_disks("c4")
    s = bench.reference_sample(disks, K, W)
    assert sum(t for _, t, _ in s) == K
    assert all(w >= 1 for _, _, w in s)
    sizes = [int(disks[k][0]["Nrad"]) for k, _, _ in s]
    assert sizes == sorted(set(sizes))
