"""The frequency-sweep workload generator (no GPU): A(w) = K - w^2 M + i w C
on the 27-point pattern, the sweep's default static-pivoting settings, and the
round-robin sharding of frequencies across ranks (two gloo ranks)."""
import numpy as np
import pytest
import scipy.sparse as sp

from rslab_b200 import matgen
from rslab_b200.solver import ZeroPivotAction
from rslab_b200.sweep import sweep_settings


def test_c4_system_structure_and_formula():
    c4 = matgen.C4System(side=8, seed=3)
    assert c4.n == 512
    K = c4.K.to_scipy_full()
    # 27-point stencil: interior rows hold 27 entries, off-diagonals are -1
    nnz_rows = (K != 0).sum(axis=1).A1
    assert nnz_rows.max() == 27 and nnz_rows.min() == 8
    off = (K - sp.diags(K.diagonal())).tocsr()
    off.eliminate_zeros()
    assert set(np.unique(off.data)) == {-1.0}
    d = K.diagonal()
    assert d.min() >= 26.0 and d.max() <= 26.1
    assert 0.5 <= c4.mdiag.min() and c4.mdiag.max() <= 1.5
    w = c4.omegas(64)
    assert len(w) == 64 and np.isclose(w[0], 0.1 * np.sqrt(c4.lambda_mid)) and np.isclose(w[-1], 2 * np.sqrt(c4.lambda_mid))
    om = w[17]
    A = c4.matrix(om).to_scipy_full()
    ref = K.astype(np.complex128) * (1 + 0.01j * om) - om * om * sp.diags(c4.mdiag)
    assert abs(A - ref).max() < 1e-12
    assert abs(A - A.T).max() == 0.0


def test_c4_matrix_is_deterministic_and_pattern_fixed():
    a = matgen.C4System(side=6, seed=3)
    b = matgen.C4System(side=6, seed=3)
    x, y = a.matrix(1.3), b.matrix(2.1)
    assert np.array_equal(x.col_ptr, y.col_ptr) and np.array_equal(x.row_idx, y.row_idx)
    assert np.array_equal(a.K.values, b.K.values) and np.array_equal(a.mdiag, b.mdiag)


def test_sweep_settings_use_static_pivoting():
    st = sweep_settings()
    assert st.on_zero_pivot == ZeroPivotAction.perturb_to_eps(1e-10)


def test_shard_frequencies_round_robin():
    from rslab_b200.sweep import shard_frequencies
    parts = [shard_frequencies(64, r, 3) for r in range(3)]
    assert sorted(i for p in parts for i in p) == list(range(64))
    assert [len(p) for p in parts] == [22, 21, 21]
    with pytest.raises(ValueError):
        shard_frequencies(8, 2, 2)


def _sweep_rank(rank, ws, port, q):
    import os

    import torch.distributed as dist

    from rslab_b200 import LdltSymbolic
    from rslab_b200.sweep import gather_certificates, shard_frequencies, sweep_settings
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        c4 = matgen.C4System(side=5, seed=3)
        om = c4.omegas(10)
        mine = shard_frequencies(len(om), rank, ws)
        # a rank's host-side share of the work: its frequencies' matrices and analyses
        rec = {}
        for i in mine:
            a = c4.matrix(om[i])
            info = LdltSymbolic.analyze_with(a, sweep_settings()).info()
            rec[i] = (float(np.abs(np.asarray(a.values)).sum()), int(info.panel_elems))
        q.put((rank, gather_certificates({"rank": rank, "records": rec}, ws)))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_sweep_gloo():
    import multiprocessing as mp
    import socket

    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sweep_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    c4 = matgen.C4System(side=5, seed=3)
    om = c4.omegas(10)
    for r in range(ws):
        merged = {}
        for part in res[r]:
            merged.update(part["records"])
        assert sorted(merged) == list(range(10))
        for i, (s1, pe) in merged.items():
            assert s1 == pytest.approx(float(np.abs(np.asarray(c4.matrix(om[i]).values)).sum()), rel=1e-15)
        assert len({pe for _, pe in merged.values()}) == 1  # one pattern, one structure
