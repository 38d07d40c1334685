"""Sharding across ranks on CPU: world_size 2 over gloo, the oracle as the per-rank compute.

The sharded RQMC driver must give the one-process result bit for bit (each replica's sums are
computed by one rank and the all-reduce adds only zeros to them), and the sharded book must
return every option's result in book order."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    import oracle_py as orc
    T = orc.T
    return orc, T.gbm(100.0, 0.03, 0.25, 1.0), T.asian(100.0)


def _oracle_pass(r0, nr, offset, n, salt_base=42, n_steps=16):
    orc, m, p = _problem()
    return orc.qmc_sums(m, p, n_steps, None, salt_base + r0, nr, offset, n, 0, 1)


def _rank_main(rank, world, port, R, eps, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from conftest import load_engine
    load_engine()
    import fdmc_b200.sharded as sh
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = sh.run_qmc_sharded(_oracle_pass, R, eps, 256, max_doublings=6)
        book = sh.price_book_sharded(lambda opts: [("priced", o, rank) for o in opts], list(range(11)))
        np.save(os.path.join(out_dir, "qmc_%d.npy" % rank),
                np.array([res["price"], res["std_error"], res["n_samples"], res["doublings"]]))
        np.save(os.path.join(out_dir, "book_%d.npy" % rank), np.array([[o, r] for _, o, r in book]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("R", [8, 5])
def test_sharded_qmc_equals_one_process(eng, tmp_path, R):
    import fdmc_b200.sharded as sh
    eps = 2e-3
    one = sh.run_qmc_sharded(_oracle_pass, R, eps, 256, max_doublings=6)   # no process group: world 1
    assert one["doublings"] >= 2
    mp.spawn(_rank_main, args=(2, _free_port(), R, eps, str(tmp_path)), nprocs=2, join=True)
    for rank in range(2):
        got = np.load(tmp_path / ("qmc_%d.npy" % rank))
        assert got[0] == one["price"] and got[1] == one["std_error"], (got, one)
        assert got[2] == one["n_samples"] and got[3] == one["doublings"]
        book = np.load(tmp_path / ("book_%d.npy" % rank))
        assert book[:, 0].tolist() == list(range(11))            # book order restored
        assert book[:, 1].tolist() == [i % 2 for i in range(11)]  # dealt round-robin


def test_sharded_qmc_matches_the_oracle_driver(eng, orc):
    """One process: the sharded loop is the oracle's own run_qmc restatement."""
    import fdmc_b200.sharded as sh
    _, m, p = _problem()
    one = sh.run_qmc_sharded(_oracle_pass, 8, 2e-3, 256, max_doublings=6)
    ref = orc.run_qmc(m, p, 2e-3, 16, None, R=8, max_doublings=6, N0=256, salt_base=42, threads=1)
    assert one["n_samples"] == ref["n_samples"]
    assert abs(one["price"] - ref["price"]) < 1e-12 and abs(one["std_error"] - ref["std_error"]) < 1e-12


def test_replica_blocks_cover_every_replica_once(eng):
    import fdmc_b200.sharded as sh
    for R in (1, 2, 5, 16, 33):
        for world in (1, 2, 3, 8):
            blocks = [sh.replica_block(R, world, k) for k in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == R
            assert all(blocks[k][1] == blocks[k + 1][0] for k in range(world - 1))
            sizes = [b - a for a, b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sh.replica_block(4, 2, 2)
    assert sh.book_share(7, 3, 1) == [1, 4]


def _oracle_level(l, r0, nr, offset, n, R=5, salt_base=42, M=2):
    import oracle_py as orc
    T = orc.T
    m, p = T.gbm(100.0, 0.05, 0.2, 1.0), T.european(100.0, 0.05, 1.0)
    return orc.level_sums(m, p, M ** l, M if l else 0, None, use_sobol=True, salt_base=salt_base + l * R + r0,
                          R=nr, offset=offset, N=n, threads=1)


def _rank_mlqmc(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from conftest import load_engine
    load_engine()
    import fdmc_b200.sharded as sh
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        r = sh.run_mlqmc_sharded(_oracle_level, 5, 2e-2, M=2, max_L=6, pilot_n=200)
        np.save(os.path.join(out_dir, "mlqmc_%d.npy" % rank),
                np.array([r["price"], r["std_error"], r["n_samples"], r["levels"], float(r["converged"])]))
    finally:
        dist.destroy_process_group()


def test_sharded_mlqmc_equals_one_process(eng, tmp_path):
    """The sharded MLQMC loop (each level's 5 replicas split 3 + 2 over two gloo ranks, one
    all-reduce per collect) gives the one-process result bit for bit when each replica's level sums
    do not depend on its launch's other replicas (the oracle's), and prices the GBM European close
    to Black-Scholes."""
    import fdmc_b200.sharded as sh
    one = sh.run_mlqmc_sharded(_oracle_level, 5, 2e-2, M=2, max_L=6, pilot_n=200)
    assert one["levels"] >= 3
    mp.spawn(_rank_mlqmc, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for rank in range(2):
        got = np.load(tmp_path / ("mlqmc_%d.npy" % rank))
        assert got[0] == one["price"] and got[1] == one["std_error"], (got, one)
        assert got[2] == one["n_samples"] and got[3] == one["levels"]
    import oracle_py as orc
    assert abs(one["price"] - orc.bs_call(100, 100, 1, 0.05, 0.2)) < 3 * one["std_error"] + 2e-2 / np.sqrt(2)


def _rank_combine(rank, world, port, R, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from conftest import load_engine
    load_engine()
    import fdmc_b200.sharded as sh
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r0, r1 = sh.replica_block(R, world, rank)
        full = np.array([[1.0 / (3 + r), np.pi * (r + 1) / 7, -r / 11.0] for r in range(R)])   # every rank knows it
        got = sh.combine_replica_sums(torch.tensor(full[r0:r1]), R)
        np.save(os.path.join(out_dir, "combine_%d.npy" % rank), got.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("R,world", [(5, 2), (2, 3)])
def test_combine_replica_sums_is_bit_exact(eng, tmp_path, R, world):
    """The benchmark's per-pass exchange: each rank's block of per-replica sums (uneven blocks, and
    an empty one when ranks outnumber replicas) becomes every replica's sums on every rank, bit for bit."""
    mp.spawn(_rank_combine, args=(world, _free_port(), R, str(tmp_path)), nprocs=world, join=True)
    full = np.array([[1.0 / (3 + r), np.pi * (r + 1) / 7, -r / 11.0] for r in range(R)])
    for rank in range(world):
        got = np.load(tmp_path / ("combine_%d.npy" % rank))
        assert np.array_equal(got, full), (rank, got, full)
