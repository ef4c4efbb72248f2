"""The multi-GPU Fock build's partition and all-reduce on CPU: N = 2 and 3
gloo ranks take the screened quartet candidates t = rank (mod N) of the
enumeration the device uses (shard.fock_candidates), digest their shares
with the oracle as the per-rank engine, and all-reduce the partial G; the
sum must equal the oracle's full G, and the shares must be disjoint,
complete and balanced."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from librint_b200 import shard
from librint_b200.basis import Molecule

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.npz")


def _molecule():
    g = np.load(GOLDEN)
    return Molecule(g["mol/h2o/def2svp/atm"], g["mol/h2o/def2svp/bas"], g["mol/h2o/def2svp/env"], 10)


def _density(m):
    n = m.nao(0)
    rng = np.random.default_rng(3)
    A = rng.standard_normal((n, n))
    return (A + A.T) / np.sqrt(n)


def _pairs(m):
    """The device's pair table order: I outer, J <= I."""
    nb = m.nbas
    return [(i, j) for i in range(nb) for j in range(i + 1)]


def _schwarz(m, pairs):
    sh = np.array([(i, j, i, j) for i, j in pairs], dtype=np.int32)
    blocks = oracle.int2e_batch(m, sh, 0)
    l = m.bas.reshape(-1, 8)[:, 1]
    nc = (l + 1) * (l + 2) // 2
    Q, o = [], 0
    for i, j in pairs:
        a, b = nc[i], nc[j]
        blk = blocks[o:o + a * b * a * b].reshape(b, a, b, a)   # [l][k][j][i]
        o += a * b * a * b
        Q.append(np.sqrt(max(abs(blk[y, x, y, x]) for x in range(a) for y in range(b))))
    return np.array(Q)


def _block_max(m, P):
    l = m.bas.reshape(-1, 8)[:, 1]
    off = np.concatenate([[0], np.cumsum((l + 1) * (l + 2) // 2)])
    nb = m.nbas
    D = np.zeros((nb, nb))
    for i in range(nb):
        for j in range(nb):
            D[i, j] = np.abs(P[off[i]:off[i + 1], off[j]:off[j + 1]]).max()
    return D


def share(m, P, tau, rank, nranks):
    """This rank's canonical quartets (screened like k_screen_sorted) and
    their distinct slots of the reference's nbas^4 loop."""
    pairs = _pairs(m)
    Q = _schwarz(m, pairs)
    D = _block_max(m, P)
    t, b, k = shard.fock_candidates(Q, D.max(), tau)
    mine = t % nranks == rank
    quartets, slots = [], set()
    for tb, kb in zip(b[mine], k[mine]):
        (I, J), (K, L) = pairs[tb], pairs[kb]
        d = max(2 * D[I, J], 2 * D[K, L], D[I, K], D[I, L], D[J, K], D[J, L])
        if Q[tb] * Q[kb] * d < tau:
            continue
        quartets.append((int(tb), int(kb)))
        for a, c in (((I, J), (K, L)), ((K, L), (I, J))):
            for x in (a, a[::-1]):
                for y in (c, c[::-1]):
                    slots.add((x[0], x[1], y[0], y[1]))
    return quartets, np.array(sorted(slots), dtype=np.int32).reshape(-1, 4)


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", world_size=world, rank=rank)
    try:
        m = _molecule()
        P = _density(m)
        quartets, slots = share(m, P, 0.0, rank, world)
        G = torch.from_numpy(oracle.fock_G_quartets(m, P, slots, nthreads=2))
        dist.all_reduce(G)                    # the per-build collective
        gathered = [None] * world
        dist.all_gather_object(gathered, quartets)
        q.put((rank, G.numpy(), gathered))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_partition_fock_build(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() * 7 + world) % 1000
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m = _molecule()
    G_full = oracle.fock_G(m, _density(m))
    npair = m.nbas * (m.nbas + 1) // 2
    for rank, G, gathered in out:
        np.testing.assert_allclose(G, G_full, rtol=1e-12, atol=1e-12 * np.abs(G_full).max())
        shares = [set(g) for g in gathered]
        for a in range(world):
            for b in range(a + 1, world):
                assert not (shares[a] & shares[b])         # disjoint
        assert len(set().union(*shares)) == npair * (npair + 1) // 2   # every quartet (tau = 0)
        sizes = [len(x) for x in shares]
        assert max(sizes) - min(sizes) <= 1                # balanced


def test_candidate_enumeration_prefix_rule():
    """Sorted position i keeps the ket positions j <= i with Q_i Q_j 2 Dmax
    >= tau (a prefix, as the Schwarz factors descend)."""
    Q = np.array([0.5, 2.0, 1.0, 0.01, 1.0])
    t, b, k = shard.fock_candidates(Q, 1.0, 0.1)
    assert list(b) == [1, 2, 2, 4, 4, 4, 0, 0, 0, 0]
    assert list(k) == [1, 1, 2, 1, 2, 4, 1, 2, 4, 0]
    assert (Q[b] * Q[k] * 2.0 >= 0.1).all()
