"""k-NN (PLD tail) against the FP64 oracle.

Distances come from the BF16 hi/lo tensor-core minus_square; outside the
cancellation band their squared value carries at most
(4 * 2^-16 + 2 * D * 2^-24) * 2 (|q|^2 + |r|^2) absolute error, inside it the
exact FP32 sum.  The checks:
  * every returned index's true (FP64) distance matches the oracle's k-th
    order statistics within that bound (the neighbour SET is right up to
    near-ties),
  * returned distances match the true distances of the returned indices,
  * at least 99 % of indices equal the oracle's (the reference's own PLD test
    asks 90 %, apps/pld/emulation/test.cpp:95-115).
"""
import numpy as np
import pytest
import torch

import oracle
import simd2_b200 as s2
from simd2_b200 import datagen

pytestmark = pytest.mark.gpu


def check(q, r, k, dist, idx):
    want_d, want_i, want_sq = oracle.knn(q, r, k)
    D = q.shape[1]
    nq = (q.astype(np.float64) ** 2).sum(1)
    nr = (r.astype(np.float64) ** 2).sum(1)
    true_sq = ((q[:, None, :].astype(np.float64) - r[idx.clip(0)].astype(np.float64)) ** 2).sum(-1)
    bound = (4 * 2.0 ** -16 + 2 * D * 2.0 ** -24) * 2 * (nq[:, None] + nr[idx.clip(0)]) + 1e-12
    assert np.all(np.abs(np.sort(true_sq, 1) - want_sq) <= bound)
    assert np.all(np.abs(dist.astype(np.float64) ** 2 - true_sq) <= bound + 1e-6 * true_sq)
    assert (idx == want_i).mean() >= 0.99
    return (idx == want_i).mean()


@pytest.mark.parametrize("shape", [(300, 1000, 128, 16), (129, 257, 37, 5), (64, 4096, 128, 32), (1, 3, 8, 3)])
def test_knn_matches_oracle(cuda, shape):
    Q, R, D, k = shape
    q, r = datagen.point_cloud(Q, R, D, seed=Q + R, dup_frac=0.05)
    dist, idx = s2.knn(torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda), min(k, R))
    check(q, r, min(k, R), dist.cpu().numpy(), idx.cpu().numpy())


def test_knn_near_duplicates_exact(cuda):
    """Queries that are reference points plus 1e-3 noise: the nearest distance
    is computed in the exact FP32 band (relative error ~1e-6, not ~1e-2)."""
    q, r = datagen.point_cloud(500, 2000, 128, seed=9, dup_frac=1.0)
    dist, idx = s2.knn(torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda), 4)
    want_d, want_i, want_sq = oracle.knn(q, r, 4)
    d0 = dist.cpu().numpy()[:, 0].astype(np.float64)
    assert np.all(idx.cpu().numpy()[:, 0] == want_i[:, 0])
    assert np.max(np.abs(d0 - np.sqrt(want_sq[:, 0])) / np.sqrt(want_sq[:, 0])) < 1e-4


def test_knn_ties_keep_lower_index(cuda):
    """Duplicate reference points: equal distances list the lower index first."""
    rng = np.random.default_rng(2)
    base = rng.standard_normal((50, 16)).astype(np.float32)
    r = np.concatenate([base, base, base])  # each point three times
    q = base[:10] + np.float32(0.5)
    dist, idx = s2.knn(torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda), 6)
    want_d, want_i, _ = oracle.knn(q, r, 6)
    np.testing.assert_array_equal(idx.cpu().numpy(), want_i)


@pytest.mark.parametrize("shape", [(300, 1000, 128, 16), (129, 257, 37, 5), (64, 4096, 128, 32), (1, 3, 8, 3),
                                   (1000, 5000, 64, 8), (257, 70001, 100, 16), (130, 512, 128, 4),
                                   (4096, 65536, 128, 16), (8192, 65536, 128, 16), (9000, 40000, 96, 8)])
def test_knn_fused_matches_materialised(cuda, shape):
    """The fused kernel (selection in the MMA epilogue) and the materialised
    path (distance blocks, then selection) return identical bits.  From
    4096 x 65536 on, units prune with the lists of finished earlier chunks;
    the last two shapes fill more than one wave, so the fused grid opens with
    a pilot chunk of four reference tiles per query block (whose lists bound
    every later unit), the second with a ragged last tile and D = 96."""
    Q, R, D, k = shape
    q, r = datagen.point_cloud(Q, R, D, seed=Q * 7 + R, dup_frac=0.05)
    Qt, Rt = torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda)
    d1, i1 = s2.knn(Qt, Rt, min(k, R), mode="fused")
    d2, i2 = s2.knn(Qt, Rt, min(k, R), mode="materialised")
    assert torch.equal(i1, i2)
    assert torch.equal(d1.view(torch.int32), d2.view(torch.int32))
    assert s2.device_status() == 0


def test_knn_fused_ties_and_fewer_refs_than_k(cuda):
    """Duplicated references across reference tiles and chunks keep the lower
    index first; with R < k the tail is +inf / -1, in both modes."""
    rng = np.random.default_rng(5)
    base = rng.standard_normal((300, 24)).astype(np.float32)
    r = np.concatenate([base] * 4)  # copies 300 apart: different 256-wide tiles
    q = base[:40] + np.float32(0.25)
    Qt, Rt = torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda)
    d, i = s2.knn(Qt, Rt, 8, mode="fused")
    _, want_i, _ = oracle.knn(q, r, 8)
    np.testing.assert_array_equal(i.cpu().numpy(), want_i)
    small = torch.from_numpy(base[:5]).to(cuda)
    d, i = s2.knn(Qt, small, 8, mode="fused")
    assert torch.all(i[:, 5:] == -1) and torch.all(torch.isinf(d[:, 5:]))
    d2, i2 = s2.knn(Qt, small, 8, mode="materialised")
    assert torch.equal(i, i2) and torch.equal(d.view(torch.int32), d2.view(torch.int32))


@pytest.mark.parametrize("D,pad,shift", [(128, 3, 1), (37, 5, 2), (64, 0, 0), (120, 4, 4)])
def test_knn_fused_strided_and_unaligned_rows(cuda, D, pad, shift):
    """Rows with a pitch past D and a base off the 16-byte boundary (the
    operand prep then loads element by element): both modes agree bit for
    bit, and with the oracle; R = 1000 leaves a ragged last reference tile."""
    Q, R, k = 300, 1000, 16
    q, r = datagen.point_cloud(Q, R, D, seed=D * 11 + pad, dup_frac=0.05)
    qb = torch.zeros((Q, D + pad + shift), dtype=torch.float32, device=cuda)
    rb = torch.zeros((R, D + pad + shift), dtype=torch.float32, device=cuda)
    qb[:, shift:shift + D] = torch.from_numpy(q).to(cuda)
    rb[:, shift:shift + D] = torch.from_numpy(r).to(cuda)
    Qt, Rt = qb[:, shift:shift + D], rb[:, shift:shift + D]
    d1, i1 = s2.knn(Qt, Rt, k, mode="fused")
    d2, i2 = s2.knn(Qt, Rt, k, mode="materialised")
    assert torch.equal(i1, i2)
    assert torch.equal(d1.view(torch.int32), d2.view(torch.int32))
    check(q, r, k, d1.cpu().numpy(), i1.cpu().numpy())
    d3, i3 = s2.knn(torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda), k, mode="fused")
    assert torch.equal(i1, i3) and torch.equal(d1.view(torch.int32), d3.view(torch.int32))
    assert s2.device_status() == 0


def test_knn_fused_rejects_wide_points(cuda):
    q = torch.zeros(4, 200, device=cuda)
    with pytest.raises(s2.Simd2Error):
        s2.knn(q, q, 2, mode="fused")
    d, i = s2.knn(q, q, 2)  # auto falls back to the materialised path
    assert torch.all(d == 0)


@pytest.mark.parametrize("k,Q", [(16, 512), (10, 512), (32, 512), (6, 512), (16, 500), (12, 500)])
def test_knn_fused_half_lists_redo_flagged_blocks(cuda, k, Q):
    """For k > 4 the fused path first keeps lists of half the size per chunk
    half and redoes, with full lists, every query block where one list may
    have been cut short.  Here the queries of blocks 1 and 3 have all their
    nearest references in one half of one reference tile (a tight cluster at
    indices 256..383), the other blocks' queries are spread out: the result
    must equal the materialised path bit for bit, with both kinds of block in
    one call, and the oracle's neighbours.  Q = 500 makes the last, clustered
    block a partial one (rows 384..499)."""
    rng = np.random.default_rng(k + Q)
    D, R = 64, 4096
    r = rng.standard_normal((R, D)).astype(np.float32) * 4
    center = rng.standard_normal(D).astype(np.float32) * 4
    r[256:384] = center + 0.05 * rng.standard_normal((128, D)).astype(np.float32)
    q = rng.standard_normal((Q, D)).astype(np.float32) * 4
    for blk in (1, 3):
        rows = min(Q, (blk + 1) * 128) - blk * 128
        q[blk * 128:blk * 128 + rows] = center + 0.05 * rng.standard_normal((rows, D)).astype(np.float32)
    Qt, Rt = torch.from_numpy(q).to(cuda), torch.from_numpy(r).to(cuda)
    d1, i1 = s2.knn(Qt, Rt, k, mode="fused")
    d2, i2 = s2.knn(Qt, Rt, k, mode="materialised")
    assert torch.equal(i1, i2)
    assert torch.equal(d1.view(torch.int32), d2.view(torch.int32))
    ii = i1.cpu().numpy()
    for lo, hi in ((128, 256), (384, Q)):  # the clustered blocks' neighbours
        assert np.all((ii[lo:hi] >= 256) & (ii[lo:hi] < 384))
    check(q, r, k, d1.cpu().numpy(), ii)
    assert s2.device_status() == 0
