"""Batches of independent instances (the sweep configuration): greedy
partition across GPUs, host-side gather on two gloo ranks, and on the GPU
the batched stepping against single contexts and the oracle."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from gelios_2d_b200 import sweep

ROOT = Path(__file__).resolve().parent.parent


def test_partition_covers_every_instance_once_and_balances():
    counts = [400_000, 50_000, 230_000, 120_000, 310_000, 75_000, 180_000, 260_000, 90_000]
    for parts in (1, 2, 3, 4, 9, 12):
        p = sweep.partition(counts, parts)
        flat = sorted(i for part in p for i in part)
        assert flat == list(range(len(counts)))
        loads = [sum(counts[i] for i in part) for part in p]
        assert max(loads) <= sum(counts) / parts + max(counts)
    assert sweep.partition(counts, 3) == sweep.partition(counts, 3)
    with pytest.raises(ValueError):
        sweep.partition(counts, 0)


def test_instance_set_is_seeded_and_uneven():
    a = sweep.instance_set(4, seed=7, scale=(0.06, 0.12))
    b = sweep.instance_set(4, seed=7, scale=(0.06, 0.12))
    assert [m.n_cells for m, *_ in a] == [m.n_cells for m, *_ in b]
    assert len({m.n_cells for m, *_ in a}) > 1
    for (ma, pa, sa, ca), (mb, pb, sb, cb) in zip(a, b):
        assert np.array_equal(sa, sb)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from gelios_2d_b200 import sweep as sw

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        counts = [5, 9, 2, 7, 4, 8, 1]
        mine = sw.partition(counts, world)[rank]
        merged = sw.gather_results({i: counts[i] * 10 for i in mine}, dist)
        if rank == 0:
            with open(os.path.join(out_dir, "merged.txt"), "w") as f:
                f.write(repr(sorted(merged.items())))
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


def test_gather_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    merged = eval((tmp_path / "merged.txt").read_text())
    assert merged == [(i, c * 10) for i, c in enumerate([5, 9, 2, 7, 4, 8, 1])]


@pytest.mark.gpu
def test_batched_instances_match_single_contexts_and_oracle():
    import gelios_2d_b200 as g
    from oracle import oracle as O

    inst = sweep.instance_set(3, seed=11, scale=(0.25, 0.35))
    B = sweep.Sweep(inst)
    B.step(3)
    for i, (mesh, params, st0, mc) in enumerate(inst):
        S = g.Setka(mesh, params)
        S.set_par(0, st0)
        S.set_par(1, st0)
        S.set_mc(*mc)
        S.Go_5_komponent__MK2(3)
        for b in (0, 1):
            assert np.array_equal(B.par(i, b), S.par(b))
    mesh, params, st0, mc = inst[0]
    d = {n: getattr(params, n) for n, _ in O.GoParams._fields_ if n != "pad_"}
    ora = O.Oracle(O.GoParams(**d, pad_=0), mesh)
    for b in (0, 1):
        ora.set_state(b, st0)
    ora.set_mc(*mc)
    ora.mk2(3)
    a, r = B.par(0, 1), ora.get_state(1)
    err = max(float(np.max(np.abs(a[k] - r[k])) / np.max(np.abs(r[k]))) for k in range(5))
    assert err <= 1e-10
    B.close()
