"""Host logic of the sharded estimator (one bispectrum over several GPUs):
the ring-triplet assignment (beam_shard_assign, a host-only library call) and
the sum-reduce of partial bins over torch.distributed, run as world_size-2
gloo ranks on the CPU.

The partial bins each rank reduces are built from the oracle's per-triangle
sums B (barbie.c:315-337) and cal_coeff weights (funcs.c:708-745) over the
triangles of the ring triplets assigned to it, following the binning of
barbie.c:343-363; their reduction must give back the oracle's whole-estimator
bins."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden_field


def test_shard_assign_longest_processing_time(beamlib):
    # 5 -> s0, 3 -> s1, 3 -> s1 (3 < 5), 2 -> s0 (5 < 6), 2 -> s1 (6 < 7), 1 -> s0 (7 < 8)
    assert beamlib.shard_assign([5, 3, 3, 2, 2, 1], 2).tolist() == [0, 1, 1, 0, 1, 0]
    # ties in work keep index order, ties in load go to the lower shard
    assert beamlib.shard_assign([1, 1, 1, 1], 4).tolist() == [0, 1, 2, 3]
    assert beamlib.shard_assign([2, 7, 7], 2).tolist() == [0, 0, 1]
    assert beamlib.shard_assign([4.0, 9.0], 1).tolist() == [0, 0]
    assert beamlib.shard_assign([], 3).tolist() == []


def test_shard_assign_balances_and_is_deterministic(beamlib):
    rng = np.random.default_rng(7)
    work = rng.integers(1, 10_000, size=1305).astype(np.float64) * rng.integers(1, 4000, size=1305)
    for k in (2, 3, 8):
        owner = beamlib.shard_assign(work, k)
        assert np.array_equal(owner, beamlib.shard_assign(work, k))
        assert owner.min() >= 0 and owner.max() < k
        load = np.bincount(owner, weights=work, minlength=k)
        # LPT bound: no shard exceeds the mean by more than the largest unit
        assert load.max() - load.mean() <= work.max() + 1e-9


def test_shard_assign_rejects_bad_arguments(beamlib):
    with pytest.raises(beamlib.BeamError) as e:
        beamlib.shard_assign([1.0, 2.0], 0)
    assert e.value.code == beamlib.BEAM_EINVAL


def _partials(data, owner_of_rp, rank):
    """Partial bins of the triangles whose ring triplet belongs to `rank`."""
    tri, B, wb, wn, nn2, shape = data["tri"], data["B"], data["wb"], data["wn"], data["nn2"], data["shape"]
    mine = owner_of_rp[tri["rp"]] == rank
    bs, norm = np.zeros(shape), np.zeros(shape)
    count = np.zeros(shape[:3], dtype=np.int64)
    nz = B != 0.0
    for t in np.flatnonzero(mine):
        i, j, l = tri["k1_bin"][t], tri["t_bin"][t], tri["mu_bin"][t]
        bs[i, j, l] += B[t] * wb[t]
        num = tri["num"][t] if nz[t] else 0.0
        norm[i, j, l] += num * wn[t]
        if nz[t]:
            count[i, j, l] += int(round(tri["num"][t] / nn2))
    return dict(bs=bs, norm=norm, count=count)


def _rank_main(rank, world, port, data, owner_of_rp, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from barbie_b200 import shard
        res = shard.allreduce_partials(_partials(data, owner_of_rp, rank), data["vol"])
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2])
def test_gloo_sharded_bins_match_the_whole_estimator(oracle, beamlib, world):
    name = "nn64_cfg1"
    NN, Nmax, Nr, UL, LL, BW, _ = GOLDEN_CASES[name]
    field = golden_field(name)
    full = oracle.estimate(field, NN, Nmax, Nr, UL, LL, BW, want_B=True)
    tri, _ = oracle.enumerate_triples(NN, Nmax, Nr, UL, LL, BW)
    nn2 = float(NN * NN)
    wb = np.zeros((len(tri), 16))
    wn = np.zeros((len(tri), 16))
    for t in range(len(tri)):
        wb[t], wn[t] = oracle.cal_coeff(tri["px"][t], tri["pz"][t])
    # work per used ring triplet (in calCR order), as the plan computes it:
    # accepted triangles x in-plane triangles
    used = np.unique(tri["rp"])
    ncombo = np.bincount(tri["rp"], minlength=used.max() + 1)[used]
    ntau = np.array([round(tri["num"][np.flatnonzero(tri["rp"] == rp)[0]] / nn2) for rp in used])
    owner = beamlib.shard_assign(ncombo.astype(np.float64) * ntau, world)
    owner_of_rp = np.full(used.max() + 1, -1, dtype=np.int64)
    owner_of_rp[used] = owner
    assert set(owner.tolist()) == set(range(world))
    data = dict(tri=tri, B=full["B"], wb=wb, wn=wn, nn2=nn2, shape=full["bs"].shape, vol=float(NN) ** 3)

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, data, owner_of_rp, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        res = got[r]
        assert np.array_equal(res["count"], full["counts"])
        for key in ("bs", "norm"):
            scale = np.maximum(np.abs(full[key]), 1e-300)
            assert np.all(np.abs(res[key] - full[key]) <= 1e-12 * scale + 1e-300), key
        ok = full["norm"][..., 0] > 0.1
        # out = bs/(vol*norm): relative errors of bs and norm add; empty (l,m) norms give NaN on both sides
        assert np.allclose(res["out"][ok], full["out"][ok], rtol=3e-12, atol=0, equal_nan=True)
    assert np.array_equal(got[0]["bs"], got[1]["bs"])  # every rank ends with the same bins
