"""bench.py's reference arm under the multi-rank launch the harness uses
(torch.distributed.run, two ranks on this host): rank 0 alone prints one JSON
line with the contract's keys, the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_under_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
           "--particles", "2"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference"
    assert rec["n_gpus"] == 2 and rec["steps"] == 1 and rec["warmup"] == 3
    assert rec["value"] > 0 and rec["higher_is_better"] is True
    for key in ("metric", "unit", "config", "cpu_baseline", "e2e"):
        assert key in rec
    assert rec["e2e"]["h2d_bytes_per_step"] == 0 and rec["e2e"]["d2h_bytes_per_step"] == 0
    assert rec["cpu_baseline"]["kind"] == "port"


def test_reference_arm_loads_only_the_oracle():
    """The reference arm builds its inputs with the oracle's gamma
    discretisation and LG table: the engine library never enters the process,
    and its config is the GPU arm's."""
    code = ("import runpy, sys, json\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',"
            " '--particles', '2']\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('LOADED', json.dumps({'engine': 'libsmccat' in maps, 'oracle': 'liboracle' in maps}))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    loaded = json.loads([l for l in out.stdout.splitlines() if l.startswith("LOADED")][0][7:])
    assert loaded == {"engine": False, "oracle": True}
    rec = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][0])
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "smc-cat_b200"))
    import bench
    from smccat import workload
    assert rec["config"] == bench.bench_config(workload.CONFIGS[2], 2, 1)
