"""The multi-rank host logic of bench.py on the CPU: two gloo ranks launched
the way torch.distributed.run launches bench.py (RANK, WORLD_SIZE,
MASTER_ADDR 127.0.0.1), checking the barrier, the max over ranks that every
timed number goes through, and that the ranks of the many-molecule line get
different molecule lists (weak scaling, no collective on the data path)."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import os, sys, json
    sys.path.insert(0, os.environ["QB_ROOT"])
    import bench
    ws, rank, local = bench.dist_setup()
    import torch.distributed as dist
    assert dist.get_backend() == "gloo", dist.get_backend()
    bench.barrier(ws)
    top = bench.max_over_ranks(float(rank + 1) * 1.5, ws)
    sizes = [int(x) for x in bench.batch_sizes(16, rank)]
    print(json.dumps({"rank": rank, "ws": ws, "max": top, "sizes": sizes}))
    dist.destroy_process_group()
""")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks():
    import json
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), QB_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda o: o["rank"])
    assert [o["ws"] for o in outs] == [2, 2]
    assert all(o["max"] == 3.0 for o in outs)
    assert outs[0]["sizes"] != outs[1]["sizes"]
    assert all(1 <= n <= 12 for o in outs for n in o["sizes"])
