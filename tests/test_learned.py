"""Learned hypothesis proposal: features, MLP training kernels, batched and
weighted RANSAC, and the gain of the trained proposal over uniform sampling.

The CPU side is oracle/learned_oracle.py (float64 restatement of the
features and of the MLP's loss and gradient; its own gradient is pinned by
finite differences here) and the reference's RANSAC through the C
restatement. GPU tests call the library through its C ABI.
"""
import numpy as np
import pytest

from oracle import learned_oracle as LO
from rvpoint_b200 import datasets as D


def _rand_params(rng):
    p = np.zeros(LO.NP, np.float32)
    p[LO.OW1:LO.OB1] = rng.normal(0, 0.6, LO.OB1 - LO.OW1)
    p[LO.OB1:LO.OW2] = rng.normal(0, 0.1, LO.MH)
    p[LO.OW2:LO.OB2] = rng.normal(0, 0.2, LO.MH * LO.MH)
    p[LO.OB2:LO.OW3] = rng.normal(0, 0.1, LO.MH)
    p[LO.OW3:LO.OB3] = rng.normal(0, 0.3, LO.MH)
    p[LO.OB3] = 0.1
    return p


def test_oracle_gradient_matches_finite_differences():
    """The oracle's analytic gradient against central differences of its
    loss (weights kept exactly representable in BF16 so that the rounding
    is the identity around them)."""
    rng = np.random.default_rng(3)
    p = LO.bf16_round(_rand_params(rng))
    feat = rng.normal(size=(64, 8))
    y = (rng.uniform(size=64) < 0.4).astype(np.float64)
    mean, std = np.zeros(8), np.ones(8)
    _, g = LO.loss_and_grad(p, mean, std, feat, y)
    # differentiate in float64 without the rounding: unpack's inputs directly
    def loss_of(q):
        W1, b1, W2, b2, w3, b3 = LO.unpack(q)
        z1 = feat @ W1.T + b1
        h1 = np.maximum(z1, 0)
        h2 = np.maximum(h1 @ W2.T + b2, 0)
        o = h2 @ w3 + b3
        return np.mean(np.maximum(o, 0) - y * o + np.log1p(np.exp(-np.abs(o))))
    q = p.astype(np.float64)
    for i in list(range(0, LO.NP, 97)) + [LO.OB3]:
        e = 1e-6
        a, b = q.copy(), q.copy()
        a[i] += e
        b[i] -= e
        fd = (loss_of(a) - loss_of(b)) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), i


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, 1.0078125 + 2 ** -9, -3.14159], np.float32)
    r = LO.bf16_round(v)
    assert r[0] == 1.0
    assert r[1] == 1.0            # halfway, even mantissa stays
    assert r[2] == 1.0078125      # above halfway rounds up
    bits = r.view(np.uint32)
    assert np.all(bits & 0xFFFF == 0)


@pytest.mark.gpu
def test_mlp_forward_and_gradients_match_cpu_oracle(gpu_ctx):
    import torch
    from rvpoint_b200.learned import PlaneScorer
    rng = np.random.default_rng(5)
    p = _rand_params(rng)
    n = 5000
    feat = rng.normal(0.5, 2.0, size=(n, 8)).astype(np.float32)
    y = (rng.uniform(size=n) < 0.3).astype(np.float32)
    mean = feat.mean(0)
    std = feat.std(0)
    s = PlaneScorer(1024, 1, ctx=gpu_ctx)
    s.set_params(p)
    s.set_norm(mean, std)
    assert np.array_equal(s.get_params(), p)
    fd = torch.from_numpy(feat).cuda()
    yd = torch.from_numpy(y).cuda()
    logits = s.forward(fd).cpu().numpy()
    # the forward pass runs on tensor cores: inputs in TF32, hidden layer 1
    # in BF16, sums in FP32. Against the oracle with the same roundings the
    # FP32 sums differ by ulps, and a hidden value whose FP32 sum lies within
    # an ulp of a BF16 rounding boundary may round the other way (a BF16 ulp,
    # 2^-8 relative, of one of 64 inputs of layer 2): 2e-3 of the logit scale
    ref_tc = LO.forward(p, mean, std, feat, tensor_core=True)
    scale = 1 + np.max(np.abs(ref_tc))
    assert np.max(np.abs(logits - ref_tc)) <= 2e-3 * scale
    assert np.percentile(np.abs(logits - ref_tc), 99) <= 2e-4 * scale
    # and against exact float64 activations: the roundings themselves
    ref = LO.forward(p, mean, std, feat)
    assert np.max(np.abs(logits - ref)) <= 2e-2 * (1 + np.max(np.abs(ref)))
    loss, g = s.gradients(fd, yd)
    # the training step runs on tensor cores too: against the oracle with the
    # same roundings (BF16 operands of the backward products) the FP32 sums
    # differ by ulps and a value within an ulp of a BF16 rounding boundary
    # may round the other way: 1e-3 of the largest component, per component
    rloss, rg = LO.loss_and_grad(p, mean, std, feat, y, tensor_core=True)
    assert abs(loss - rloss) <= 1e-4 * max(1.0, abs(rloss))
    scale = np.max(np.abs(rg))
    assert np.max(np.abs(g - rg)) <= 1e-3 * scale
    # against exact float64 activations: the roundings themselves (BF16 has
    # 8 significant bits: 2^-9 relative per operand)
    eloss, eg = LO.loss_and_grad(p, mean, std, feat, y)
    assert abs(loss - eloss) <= 5e-3 * max(1.0, abs(eloss))
    assert np.max(np.abs(g - eg)) <= 2e-2 * np.max(np.abs(eg))
    s.close()


@pytest.mark.gpu
def test_training_lowers_the_loss(gpu_ctx):
    import torch
    from rvpoint_b200.learned import PlaneScorer
    rng = np.random.default_rng(9)
    n = 20000
    feat = rng.normal(size=(n, 8)).astype(np.float32)
    y = ((feat[:, 3] + 0.5 * feat[:, 5]) < 0).astype(np.float32)  # learnable rule
    s = PlaneScorer(1024, 1, ctx=gpu_ctx)
    s.set_norm(np.zeros(8, np.float32), np.ones(8, np.float32))
    fd, yd = torch.from_numpy(feat).cuda(), torch.from_numpy(y).cuda()
    first = s.train_step(fd, yd, 3e-3, want_loss=True)
    for _ in range(200):
        s.train_step(fd, yd, 3e-3)
    last, _ = s.gradients(fd, yd)
    assert last < 0.3 * first
    pred = s.forward(fd).cpu().numpy() > 0
    assert (pred == (y > 0)).mean() > 0.97
    s.close()


@pytest.mark.gpu
def test_training_is_deterministic(gpu_ctx):
    """The blocks' gradient shares are added in block order (no float
    atomics): the same data, start and seeds give bit-identical weights."""
    import torch
    from rvpoint_b200.learned import PlaneScorer
    rng = np.random.default_rng(10)
    n = 50000
    feat = rng.normal(size=(n, 8)).astype(np.float32)
    y = (feat[:, 2] > 0.3).astype(np.float32)
    fd, yd = torch.from_numpy(feat).cuda(), torch.from_numpy(y).cuda()
    out = []
    for _ in range(2):
        s = PlaneScorer(n, 1, ctx=gpu_ctx)
        s.set_norm(np.zeros(8, np.float32), np.ones(8, np.float32))
        s.set_params(rng_params := np.random.default_rng(3).normal(
            scale=0.1, size=s.get_params().shape).astype(np.float32))
        for k in range(20):
            s.train_step(fd, yd, 3e-3, batch=8192, seed=k + 1)
        loss, g = s.gradients(fd, yd)
        out.append((s.get_params(), g, loss))
        s.close()
    assert np.array_equal(out[0][0].view(np.int32), out[1][0].view(np.int32))
    assert np.array_equal(out[0][1].view(np.int32), out[1][1].view(np.int32))
    assert out[0][2] == out[1][2]
    del rng_params


@pytest.mark.gpu
def test_features_match_cpu_oracle(gpu_ctx):
    import torch
    from rvpoint_b200.learned import DeviceBatch, PlaneScorer
    scenes = [D.plane_scene(9100 + s, n=3000) for s in range(2)]
    xs = np.concatenate([c.x for c, _ in scenes])
    ys = np.concatenate([c.y for c, _ in scenes])
    zs = np.concatenate([c.z for c, _ in scenes])
    offs = np.array([0, 3000, 6000], np.int64)
    b = DeviceBatch.from_host(D.Batch(xs, ys, zs, offs))
    s = PlaneScorer(b.n, 2, ctx=gpu_ctx)
    cand = torch.arange(0, b.n, 3, dtype=torch.int32, device="cuda")
    feat = s.features(b, 1.0, cand).cpu().numpy()
    ci = cand.cpu().numpy()
    ref = []
    for f in range(2):
        a, e = offs[f], offs[f + 1]
        nb = LO.brute_knn(xs[a:e], ys[a:e], zs[a:e], 17)
        ff = LO.features(xs[a:e], ys[a:e], zs[a:e], nb)
        ref.append(ff)
    ref = np.concatenate(ref)[ci]
    err = np.abs(feat - ref)
    # FP32 shifted sums and a 6-sweep Jacobi against float64 eigh
    assert np.percentile(err[:, [3, 5, 7]], 99) < 1e-3
    assert np.percentile(err, 95) < 1e-2
    assert np.mean(err.max(1) < 5e-2) > 0.98
    s.close()


@pytest.mark.gpu
def test_features_among_candidates_equal_features_of_their_subcloud(gpu_ctx):
    import torch
    from rvpoint_b200.learned import DeviceBatch, PlaneScorer, candidates
    tr = D.plane_batch(n_scenes=3, n=20_000, seed=D.SEED_BASE + 77)
    b = DeviceBatch.from_host(tr)
    cand_h, coffs_h = candidates(b.offsets_host, 1500, 3)
    sub = D.Batch(tr.x[cand_h], tr.y[cand_h], tr.z[cand_h], coffs_h)
    s = PlaneScorer(b.n, 3, ctx=gpu_ctx)
    cand = torch.from_numpy(cand_h.view(np.int32)).cuda()
    coffs = torch.from_numpy(coffs_h).cuda()
    sb = DeviceBatch.from_host(sub)
    f2 = s.features(sb, 1.0).cpu().numpy()
    # among the candidates: two blocks per scene, each with the scene's grid
    # in shared memory
    for cell in (0.5, 1.0, 2.5):
        f1 = s.features(b, cell, cand, coffs, among_candidates=True).cpu().numpy()
        assert np.array_equal(f1.view(np.int32), f2.view(np.int32)), cell
    # the bench's scene generator at its candidate count, twice in a row at
    # each cell: 1.0 m (about one candidate per cell: rings of two and three
    # cells), 2.0 and 2.5 m (about 5 and 8 candidates per cell: mostly
    # finished at ring 1, a few queries on ring 2)
    ev = D.plane_batch(n_scenes=16, seed=D.SEED_BASE + 4)
    be = DeviceBatch.from_host(ev)
    ch, co = candidates(be.offsets_host, 1024, 11)
    se = PlaneScorer(be.n, 16, ctx=gpu_ctx)
    ref = se.features(DeviceBatch.from_host(D.Batch(ev.x[ch], ev.y[ch], ev.z[ch], co)),
                      1.0).cpu().numpy()
    for cell in (1.0, 1.0, 2.0, 2.0, 2.5, 2.5):
        fe = se.features(be, cell, torch.from_numpy(ch.view(np.int32)).cuda(),
                         torch.from_numpy(co).cuda(), among_candidates=True).cpu().numpy()
        assert np.array_equal(fe.view(np.int32), ref.view(np.int32)), cell
    se.close()
    # the batched grid kNN over the subcloud in its cooperative mode (dense
    # cells together, the rest one query per thread) finds the same neighbours
    for rfac in (0.7, 1.0, 2.0):
        for cell in (1.0, 2.5):
            s.set_knn(3, rfac)
            f3 = s.features(sb, cell).cpu().numpy()
            s.set_knn(0)
            assert np.array_equal(f3.view(np.int32), f2.view(np.int32)), (rfac, cell)
    s.close()


@pytest.mark.gpu
def test_batched_ransac_matches_reference_per_frame(gpu_ctx, restatement):
    import torch
    from oracle.oracle import libc_rand_stream
    from rvpoint_b200.learned import DeviceBatch, ransac_frames
    scenes = [D.plane_scene(9200 + s, n=6000) for s in range(3)]
    xs = np.concatenate([c.x for c, _ in scenes])
    ys = np.concatenate([c.y for c, _ in scenes])
    zs = np.concatenate([c.z for c, _ in scenes])
    offs = np.array([0, 6000, 12000, 18000], np.int64)
    b = DeviceBatch.from_host(D.Batch(xs, ys, zs, offs))
    models, best, iters = ransac_frames(b, 3000, 0.02, ctx=gpu_ctx)
    models, best, iters = models.cpu().numpy(), best.cpu().numpy(), iters.cpu().numpy()
    rs = libc_rand_stream(9000)
    for f in range(3):
        c, _ = scenes[f]
        rb, rm, _, _, rit = restatement.ransac_plane(c, 0.02, 3000, rs)
        assert best[f] == rb
        assert iters[f] == rit
        assert np.array_equal(models[f].view(np.int32), rm.view(np.int32))
    # with targets: the first hypothesis reaching the target stops the frame
    tg = torch.tensor([int(v) // 2 for v in best], dtype=torch.int32, device="cuda")
    _, b2, it2 = ransac_frames(b, 3000, 0.02, targets=tg, ctx=gpu_ctx)
    for f in range(3):
        c, _ = scenes[f]
        _, _, counts, _, _ = restatement.ransac_plane(c, 0.02, 3000, rs, prob=0.9999)
        first = int(np.argmax(counts >= int(tg[f])))
        assert int(it2[f]) == first + 1
        assert int(b2[f]) >= int(tg[f])


def _recount(c, m, t):
    x, y, z = (np.asarray(v, np.float32) for v in (c.x, c.y, c.z))
    m = np.asarray(m, np.float32)
    d = ((m[0] * x + m[1] * y) + m[2] * z) + m[3]
    return int(np.sum(np.abs(d.astype(np.float32)) <= np.float32(t)))


@pytest.mark.gpu
def test_weighted_ransac_counts_are_exact(gpu_ctx):
    import torch
    from rvpoint_b200.learned import DeviceBatch, ransac_weighted
    scenes = [D.plane_scene(9300 + s, n=8000) for s in range(3)]
    xs = np.concatenate([c.x for c, _ in scenes])
    ys = np.concatenate([c.y for c, _ in scenes])
    zs = np.concatenate([c.z for c, _ in scenes])
    offs = np.array([0, 8000, 16000, 24000], np.int64)
    b = DeviceBatch.from_host(D.Batch(xs, ys, zs, offs))
    cand = torch.arange(0, b.n, dtype=torch.int32, device="cuda")
    coffs = torch.from_numpy(offs).cuda()
    # weight plane points 1, outliers 0.05
    lab = np.concatenate([l for _, l in scenes])
    w = torch.from_numpy(np.where(lab >= 0, 1.0, 0.05).astype(np.float32)).cuda()
    models, best, iters = ransac_weighted(b, cand, coffs, w, 200, 0.02, seed=5, ctx=gpu_ctx)
    models, best = models.cpu().numpy(), best.cpu().numpy()
    for f in range(3):
        assert best[f] > 0
        assert _recount(scenes[f][0], models[f], 0.02) == best[f]
    # deterministic for a seed
    m2, b2, _ = ransac_weighted(b, cand, coffs, w, 200, 0.02, seed=5, ctx=gpu_ctx)
    assert np.array_equal(b2.cpu().numpy(), best)
    # zero weights everywhere: no hypothesis, count 0
    _, b0, _ = ransac_weighted(b, cand, coffs, torch.zeros_like(w), 50, 0.02, ctx=gpu_ctx)
    assert np.all(b0.cpu().numpy() == 0)


@pytest.mark.gpu
def test_preemptive_rounds_count_exactly_and_stop_at_targets(gpu_ctx):
    import torch
    from rvpoint_b200.learned import DeviceBatch, candidates, ransac_preemptive
    tr = D.plane_batch(n_scenes=4, n=20_000, seed=D.SEED_BASE + 91)
    b = DeviceBatch.from_host(tr)
    cand_h, coffs_h = candidates(b.offsets_host, 1024, 5)
    cand = torch.from_numpy(cand_h.view(np.int32)).cuda()
    coffs = torch.from_numpy(coffs_h).cuda()
    w = torch.ones(cand.numel(), dtype=torch.float32, device="cuda")
    models, best, drawn = ransac_preemptive(b, cand, coffs, w, 0.02, draws=128, max_rounds=3,
                                            seed=9, ctx=gpu_ctx)
    models, best, drawn = models.cpu().numpy(), best.cpu().numpy(), drawn.cpu().numpy()
    for f in range(4):
        assert best[f] > 0
        assert _recount(tr.frame(f), models[f], 0.02) == best[f]
        assert drawn[f] == 128 + 2 * 2 * 128  # later rounds draw twice the first
    tg = torch.from_numpy((best // 2).astype(np.int32)).cuda()
    _, b2, d2 = ransac_preemptive(b, cand, coffs, w, 0.02, draws=128, max_rounds=3, seed=9,
                                  targets=tg, ctx=gpu_ctx)
    assert np.all(b2.cpu().numpy() >= best // 2)
    d2 = d2.cpu().numpy()  # whole rounds, stopping at the round that reached the target
    assert np.all(np.isin(d2, [128, 128 + 256, 128 + 512]))


@pytest.mark.gpu
def test_trained_proposal_needs_fewer_hypotheses(gpu_ctx):
    """Trained on held-out scenes, the learned proposal reaches 99% of the
    plain 10k-hypothesis best count with fewer hypotheses than uniform
    sampling on fresh scenes."""
    import torch
    from rvpoint_b200.learned import (DeviceBatch, LearnedRansac, PlaneScorer, TrainConfig,
                                      ransac_frames, train)
    tr = D.plane_batch(n_scenes=24, n=50_000, seed=D.SEED_BASE + 40)
    ev = D.plane_batch(n_scenes=12, n=50_000, seed=D.SEED_BASE + 41)
    bt, be = DeviceBatch.from_host(tr), DeviceBatch.from_host(ev)
    s = PlaneScorer(max(bt.n, be.n), 24, ctx=gpu_ctx)
    info = train(s, bt, TrainConfig(steps=300))
    assert info["losses"][-1][1] < info["losses"][0][1]
    _, best, _ = ransac_frames(be, 10_000, 0.02, ctx=gpu_ctx)
    tg = torch.ceil(best.double() * 0.99).to(torch.int32)
    _, bp, itp = ransac_frames(be, 10_000, 0.02, targets=tg, ctx=gpu_ctx)
    lr = LearnedRansac(s, preemptive=False)
    cand, coffs = lr.prepare(be)
    _, bl, itl = lr.run(be, cand, coffs, 10_000, 0.02, targets=tg)
    reached = (bl >= tg).float().mean().item()
    assert reached >= 0.9
    # the preemptive rounds reach the same targets
    _, bp2, _ = LearnedRansac(s).run(be, cand, coffs, 10_000, 0.02, targets=tg)
    assert (bp2 >= tg).float().mean().item() >= 0.9
    # typical scene: the median over scenes (a scene whose best plane the
    # proposal misses falls back to the hypothesis budget)
    assert itl.double().median().item() < itp.double().median().item()
    s.close()
