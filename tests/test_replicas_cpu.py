"""Multi-GPU plan of the pass is replicas only (a frame does not shard; instances do): each rank
renders its own instance with no data-path collective, and the job time is the max over ranks.
Exercised here with two gloo ranks on CPU driving the oracle."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import datetime
    import time
    import torch.distributed as dist
    import bench
    import oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    oracle._abi()
    import reservoir_splatting_b200.scenes as S
    oracle.set_threads(1)
    p = oracle.OraclePass({"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 1}, 16, 16)
    p.set_scene(S.cornell_box(0))
    t0 = time.perf_counter()
    for f in range(3):
        img = p.execute(S.cornell_camera(f + bench.rank_frame_offset(rank) // 97 * 5, 16, 16))
    ms = (time.perf_counter() - t0) * 1e3 + 1000.0 * rank  # rank 1 is made the slowest
    job_ms = bench.max_over_ranks(ms, dist)
    np.savez(Path(out_dir) / f"rank{rank}.npz", img=img, ms=ms, job_ms=job_ms)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_render_independent_replicas(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0, r1 = np.load(tmp_path / "rank0.npz"), np.load(tmp_path / "rank1.npz")
    assert float(r0["job_ms"]) == pytest.approx(max(float(r0["ms"]), float(r1["ms"])))
    assert float(r1["job_ms"]) == float(r0["job_ms"])
    assert not np.array_equal(r0["img"], r1["img"])  # different camera-path phases
    assert np.isfinite(r0["img"]).all() and np.isfinite(r1["img"]).all()
