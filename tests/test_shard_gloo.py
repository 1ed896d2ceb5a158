"""Multi-rank logic of the build on CPU: two gloo ranks take disjoint Sobol
ranges (scp3_b200.shard), accumulate with the oracle standing in for the
device, and the all-reduced matrix must equal one process's build over the
union of the ranges (strong scaling) or over both weak-scaling ranges."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_hbuild_case


def _worker(rank, world, port, scaling, out):
    import torch
    import torch.distributed as dist
    import oracle
    from scp3_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    c = load_hbuild_case("dimer_qtip4pf")
    i0, n = shard.sample_range(rank, world, 0, 300, scaling)
    normals = oracle.std_normals(12, i0, n, scramble_seed=0x5C3)
    q, v = oracle.samples(0, 2, c["x0"], c["MUa"], c["omega"], normals)
    M = oracle.accumulate(q[:, c["modes"]], v, 12, 4)
    T = torch.from_numpy(np.ascontiguousarray(M))
    shard.reduce_matrix(T)
    if rank == 0:
        np.save(out, T.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("scaling", ["strong", "weak"])
def test_two_rank_build_equals_single(tmp_path, scaling):
    import oracle
    from scp3_b200 import shard
    out = str(tmp_path / "M.npy")
    port = 29500 + (os.getpid() % 1000) + (0 if scaling == "strong" else 1000)
    mp.start_processes(_worker, args=(2, port, scaling, out), nprocs=2, start_method="spawn", join=True)
    M2 = np.load(out)
    c = load_hbuild_case("dimer_qtip4pf")
    ranges = [shard.sample_range(r, 2, 0, 300, scaling) for r in range(2)]
    normals = np.concatenate([oracle.std_normals(12, i0, n, scramble_seed=0x5C3) for i0, n in ranges])
    q, v = oracle.samples(0, 2, c["x0"], c["MUa"], c["omega"], normals)
    M1 = oracle.accumulate(q[:, c["modes"]], v, 12, 4)
    A = oracle.accumulate(q[:, c["modes"]], v, 12, 4, absolute=True)
    assert np.all(np.abs(M2 - M1) <= 1e-13 * A + 1e-300)
    if scaling == "strong":
        assert ranges == [(0, 150), (150, 150)]
    else:
        assert ranges == [(0, 300), (1 << 40, 300)]


def test_sample_ranges_partition():
    from scp3_b200 import shard
    for world in (1, 2, 3, 8):
        rs = [shard.sample_range(r, world, 7, 1001, "strong") for r in range(world)]
        assert rs[0][0] == 7 and sum(n for _, n in rs) == 1001
        assert all(rs[k][0] + rs[k][1] == rs[k + 1][0] for k in range(world - 1))
    with pytest.raises(ValueError):
        shard.sample_range(2, 2, 0, 10)
