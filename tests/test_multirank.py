"""The multi-rank plumbing of bench.py on the CPU: world_size-2 `gloo` ranks
take the max over ranks of their timings, and under torchrun the reference
arm runs on rank 0 alone (the other rank exits 0 without output)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    mine = 10.0 + 5.0 * rank  # rank 1 is the slow one
    got = bench.max_over_ranks(mine, dist, "cpu")
    dist.barrier()
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(repr(got))
    dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    vals = [float(open(os.path.join(tmp_path, f"r{r}.txt")).read()) for r in range(2)]
    assert vals == [15.0, 15.0]


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_reference_arm_rank0_only():
    sys.path.insert(0, ROOT)
    from oracle import refimpl
    if not refimpl.available() and not refimpl.sources_present():
        pytest.skip("reference library not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c2c1024",
           "--gpus", "2", "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0


def test_batch_slices_cover_the_batch():
    sys.path.insert(0, ROOT)
    from fastandfourier_b200.shard import batch_slice
    for batch in (0, 1, 7, 256, 8193):
        for world in range(1, 9):
            sl = [batch_slice(batch, r, world) for r in range(world)]
            assert sl[0][0] == 0 and sl[-1][1] == batch
            assert all(sl[r][1] == sl[r + 1][0] for r in range(world - 1))
            sizes = [e - s for s, e in sl]
            assert max(sizes) - min(sizes) <= 1


def _split_main(rank, world, port, out_dir):
    """Each rank transforms its contiguous slice of one seeded batch with the
    CPU oracle; rank 0 gathers the slices."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from fastandfourier_b200.shard import gather, local_part
    from oracle import orc
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    batch, n = 7, 1000
    rng = np.random.default_rng(12)
    re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
    yr, yi = orc.c2c(local_part(re, rank, world), local_part(im, rank, world))
    part = torch.from_numpy(np.stack([yr, yi], axis=1))  # (slice, 2, n)
    whole = gather(part, batch, rank, world, dist)
    if rank == 0:
        np.save(os.path.join(out_dir, "gathered.npy"), whole.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_batch_split_over_ranks_gloo(tmp_path):
    """Two gloo ranks each transform a contiguous slice (4 and 3 of 7
    transforms); the gathered slices equal the whole-batch transform."""
    import numpy as np
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from oracle import orc
    port = _free_port()
    mp.start_processes(_split_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(os.path.join(tmp_path, "gathered.npy"))
    rng = np.random.default_rng(12)
    re = rng.uniform(-1, 1, (7, 1000)).astype(np.float32)
    im = rng.uniform(-1, 1, (7, 1000)).astype(np.float32)
    wr, wi = orc.c2c(re, im)
    assert np.array_equal(got[:, 0], wr) and np.array_equal(got[:, 1], wi)
