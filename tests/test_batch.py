"""Independent systems as one analysis (rslab_analyze_batch) and their
sharding across ranks.  CPU: the merged analysis equals the per-system
analyses (offset), the shard assignment is a deterministic balanced
partition, and a two-rank gloo run covers every system exactly once with the
per-system statistics gathered on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rslab_b200 import LdltSymbolic, matgen
from rslab_b200.batch import BatchSystems, analyze_batch, batch_layout, gather_stats, shard_by_weight


def small_batch():
    return [matgen.c3_matrix(5), matgen.c1_matrix(9), matgen.c3_matrix(7), matgen.c1_matrix(4)]


def test_batch_analysis_is_the_offset_union_of_single_analyses():
    systems = small_batch()
    b = BatchSystems(systems)
    sym = analyze_batch(b)
    seg, nz = batch_layout(sym)
    assert list(seg) == list(b.seg) and list(nz) == list(b.nz)
    e = sym.export()
    singles = [LdltSymbolic.analyze(a).export() for a in systems]
    # supernodes of system i follow those of system i-1, columns shifted
    first = np.concatenate([s["sn_first"] + off for s, off in zip(singles, b.seg[:-1])])
    assert np.array_equal(e["sn_first"], first)
    assert np.array_equal(e["sn_ncol"], np.concatenate([s["sn_ncol"] for s in singles]))
    assert np.array_equal(e["sn_nrow"], np.concatenate([s["sn_nrow"] for s in singles]))
    assert np.array_equal(e["sn_level"], np.concatenate([s["sn_level"] for s in singles]))
    assert np.array_equal(e["perm"], np.concatenate([s["perm"] + off for s, off in zip(singles, b.seg[:-1])]))
    assert sym.n_levels() == max(LdltSymbolic.analyze(a).n_levels() for a in systems)
    inf = sym.info()
    assert inf.flops_model == pytest.approx(sum(LdltSymbolic.analyze(a).info().flops_model for a in systems))


def test_batch_matrix_and_rhs_layout():
    systems = small_batch()
    b = BatchSystems(systems)
    m = b.as_matrix()
    m.validate()
    assert m.n == b.total_n and m.nnz == int(b.nz[-1])
    rhs = [np.full((a.n, 2), i, float) for i, a in enumerate(systems)]
    x = b.stack_rhs(rhs)
    parts = b.split(x)
    assert all(np.array_equal(p, r) for p, r in zip(parts, rhs))


def test_shard_by_weight_partition():
    w = [float(s) ** 6 for s in matgen.c3_sides(64, 2)]
    for ws in (1, 2, 3, 8):
        sh = shard_by_weight(w, ws)
        flat = sorted(i for part in sh for i in part)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in part) for part in sh]
        assert max(loads) - min(loads) <= max(w) + 1e-9
        assert sh == shard_by_weight(w, ws)


def test_c3_sides_in_range():
    s = matgen.c3_sides(512, 2)
    assert len(s) == 512 and min(s) >= 12 and max(s) <= 40
    assert len(set(s)) == 29


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank_main(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        sides = matgen.c3_sides(24, 2, 4, 9)
        mine = shard_by_weight([float(s) ** 6 for s in sides], ws)[rank]
        # the work of a rank: its systems only (here the host analysis)
        systems = [matgen.c3_matrix(sides[i]) for i in mine]
        sym = analyze_batch(BatchSystems(systems))
        local = {"rank": rank, "systems": mine, "flops": sym.info().flops_model}
        allst = gather_stats(local, ws)
        q.put((rank, allst))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_batch_gloo():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sides = matgen.c3_sides(24, 2, 4, 9)
    total = sum(LdltSymbolic.analyze(matgen.c3_matrix(s)).info().flops_model for s in sides)
    for r in range(ws):
        stats = res[r]
        assert [s["rank"] for s in stats] == [0, 1]
        covered = sorted(i for s in stats for i in s["systems"])
        assert covered == list(range(24))
        assert sum(s["flops"] for s in stats) == pytest.approx(total)
