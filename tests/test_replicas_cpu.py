"""Multi-process plumbing of bench.py on CPU: two gloo ranks (torchrun on
127.0.0.1) run the replica aggregation the GPU bench uses with NCCL.  The
path does not shard (one lattice per GPU, replicas only), so the only
collectives are the barriers and the max over ranks of the timed region."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r'''
import json, os, sys
sys.path.insert(0, {root!r})
import bench
world, rank, local = bench.dist_setup(2)
assert world == 2
bench.barrier(world)
# replica `rank` took 1 + rank seconds for 10 steps of a 1000-cell lattice
t, mlups = bench.replica_mlups(1000, 10, 1.0 + rank, world)
bench.barrier(world)
import torch.distributed as dist
assert dist.get_backend() == "gloo"
dist.destroy_process_group()
# one file per rank: two ranks printing to one pipe can interleave their lines
with open(os.path.join({out!r}, f"rank{{rank}}.json"), "w") as f:
    json.dump({{"rank": rank, "t": t, "mlups": mlups}}, f)
'''


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_replica_mlups_takes_the_slowest_rank(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT.format(root=ROOT, out=str(tmp_path)))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(script)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    assert sorted(d["rank"] for d in lines) == [0, 1]
    for d in lines:
        assert d["t"] == 2.0  # the slower replica sets the job time
        assert abs(d["mlups"] - 1000 * 10 * 2 / 2.0 / 1e6) < 1e-12  # both replicas' cells count


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_mlups(1000, 10, 0.5, 1) == (0.5, 1000 * 10 / 0.5 / 1e6)


def test_clock_summary_reads_nvidia_smi_rows():
    """The sampler's fallback parses `nvidia-smi --format=csv,noheader,nounits`
    rows and reports the median SM clock and every throttle reason seen."""
    sys.path.insert(0, ROOT)
    import bench

    class FakeProc:
        def terminate(self):
            pass

        def communicate(self, timeout=None):
            rows = ["0, 1965, 1965, 390.5, 0x0, Not Active, Not Active, Not Active, Not Active",
                    "0, 1800, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active",
                    "0, 1965, 1965, 401.0, 0x0, Not Active, Not Active, Not Active, Not Active",
                    "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
            return "\n".join(rows) + "\n", ""

    c = bench.ClockSampler(0)
    c.source, c.proc = "nvidia-smi", FakeProc()
    c.__exit__(None, None, None)
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_min_mhz"] == 1800.0
    assert s["sm_max_mhz"] == 1965.0 and s["power_w_max"] == 998.0
    assert s["reasons"] == ["sw_power_cap"]
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]
