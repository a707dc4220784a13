"""Sharding one molecule over ranks: the slices tile the packed vector, every integral's slice
is the one of its highest shell, and two gloo ranks on the CPU assemble the full vector from
their slices (the oracle stands in for each rank's device compute here; the GPU test runs
the shard plans themselves)."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
import __graft_entry__  # noqa: E402  (spawned ranks import this module without conftest)

mi = __graft_entry__.load_package()


def _bases():
    f = mi.basis.synthetic_molecule(31, 2, 3, mi.basis.POLARISED_C, mi.basis.POLARISED_H, 0.1, 1e4,
                                    "f", heavy_extra=[(3, 1)])
    return [mi.config0(), mi.config2(), mi.config1(), f, mi.build_basis(mi.h2())]


@pytest.mark.parametrize("nshards", [1, 2, 3, 4, 8])
def test_shard_ranges_tile_the_vector(nshards):
    from molints_b200 import shard
    for sh in _bases():
        rs = shard.shard_ranges(sh, nshards)
        assert rs[0][0] == 0 and rs[-1][1] == sh.npacked
        for (a, b), (c, d) in zip(rs, rs[1:]):
            assert b == c and a <= b
        # boundaries sit at tri(tri(first function of a shell))
        starts = {int(f) * (int(f) + 1) // 2 for f in sh.fn_offsets()}
        for lo, _ in rs:
            t = int((np.sqrt(8 * lo + 1) - 1) // 2)
            assert t * (t + 1) // 2 == lo and t in starts


def test_integral_owner_is_highest_shell():
    from molints_b200 import shard
    sh = mi.config2()
    n = 4
    rs = shard.shard_ranges(sh, n)
    fs = shard.shell_of_function(sh)
    rng = np.random.default_rng(0)
    for _ in range(300):
        i, j, k, l = (int(x) for x in rng.integers(0, sh.nbf, 4))
        r = shard.owner_of(sh, n, i, j, k, l)
        top = max(fs[[i, j, k, l]])
        lo_f = sh.fn_offsets()[top]
        lo = (lo_f * (lo_f + 1) // 2) * (lo_f * (lo_f + 1) // 2 + 1) // 2
        assert rs[r][0] <= lo < rs[r][1]  # the shard's shell range holds the top shell


def test_no_starved_shard():
    """Config 1 over 4 shards: every slice holds at least a quarter of the mean share."""
    from molints_b200 import shard
    sh = mi.config1()
    rs = shard.shard_ranges(sh, 4)
    sizes = np.array([hi - lo for lo, hi in rs], dtype=float)
    assert sizes.min() > 0.25 * sizes.mean()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, result_path):
    import torch
    import torch.distributed as dist
    m = mi
    from molints_b200 import shard
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sh = m.config2()
        lo, hi = shard.shard_ranges(sh, world)[rank]
        full = O.eri_packed_hgp(sh, nthreads=2)  # stand-in for this rank's device compute
        local = torch.from_numpy(full[lo:hi].copy())
        got = shard.gather_slices(local, sh)
        ok = bool(np.array_equal(got.numpy(), full))
        flag = torch.tensor([1 if ok else 0])
        dist.all_reduce(flag, op=dist.ReduceOp.MIN)
        if rank == 0:
            Path(result_path).write_text(str(int(flag.item())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_assemble_slices(tmp_path):
    import torch.multiprocessing as mp
    res = tmp_path / "ok.txt"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(res)), nprocs=2, join=True,
                       start_method="spawn")
    assert res.read_text() == "1"


@pytest.mark.gpu
def test_shard_plans_reassemble_the_vector():
    """Every shard plan run on one GPU, slices concatenated: equal to the whole-molecule plan
    within 1e-12 Eh (same-class quartets may swap bra and ket between the two orders)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from molints_b200 import engine, shard
    eng = engine.Engine(0)
    try:
        for sh in (mi.config2(), _bases()[3]):
            full = eng.eri_packed(sh)
            for n in (2, 3, 5):
                parts = []
                for r, (lo, hi) in enumerate(shard.shard_ranges(sh, n)):
                    out = torch.full((max(hi - lo, 1),), float("nan"), dtype=torch.float64, device="cuda")
                    plan, (plo, phi) = shard.compute_shard(eng, sh, r, n, out.data_ptr())
                    assert (plo, phi) == (lo, hi) and plan.npacked == hi - lo
                    torch.cuda.synchronize()
                    parts.append(out[:hi - lo].cpu().numpy())
                    plan.close()
                got = np.concatenate(parts)
                assert got.shape == full.shape and not np.isnan(got).any()
                assert np.max(np.abs(got - full)) < 1e-12
    finally:
        eng.close()
