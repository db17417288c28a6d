"""The replica plumbing of bench.py on CPU: world size 2 over gloo (127.0.0.1).

Ranks share nothing on the data path; the only collectives are the barriers
around the timed region and the max over ranks of the device time, from which
the whole-job value is units of all ranks / the slowest rank's time."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, {root!r})
    import bench
    d = bench.Dist()
    d.init()
    d.barrier()
    t = 10.0 + 5.0 * d.rank          # this rank's 'device time'
    slowest = d.max(t)
    fastest = -d.max(-t)
    units = 1000                      # each rank's units
    value = d.world * units / slowest
    d.barrier()
    d.close()
    print(json.dumps({{"rank": d.rank, "world": d.world, "slowest": slowest, "fastest": fastest, "value": value}}))
""")


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_agree_on_the_slowest_rank(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT.format(root=ROOT))
    port = _port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), OBVH_DIST_BACKEND="gloo", CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(out.strip().splitlines()[-1])
    import json
    res = [json.loads(o) for o in outs]
    for r in res:
        assert r["world"] == 2
        assert r["slowest"] == 15.0 and r["fastest"] == 10.0
        assert abs(r["value"] - 2 * 1000 / 15.0) < 1e-9


def test_reference_arm_other_ranks_exit_without_work(tmp_path):
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", OBVH_DIST_BACKEND="gloo",
               CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "dito",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""
