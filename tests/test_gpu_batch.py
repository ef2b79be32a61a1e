"""Multi-scene batch runs (sg_batcher): each batch's results are exactly those
of the same query on its scene alone, whatever shares the run.

Scenes of both widths and both node formats share runs of uneven batches
(empty, single-ray, slices of a larger ray block, closest and any hit); every
batch is compared bit for bit with GetIntersect / GetAttenuation on its scene,
and the FP32 batches also with SORT's own results through the oracle.
"""
import numpy as np
import pytest

from conftest import same_bits

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def world():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sort_b200 import Obvh, Qbvh, scenes
    specs = [(8, 0, scenes.sphere_field(8, 2, seed=1)), (4, 0, scenes.sphere_field(16, 3, seed=2)),
             (8, 1, scenes.sphere_field(12, 3, seed=3)), (4, 1, scenes.sphere_field(6, 2, seed=4))]
    accs = []
    for width, fmt, tri in specs:
        a = (Qbvh if width == 4 else Obvh)(node_format=fmt)
        a.Build(tri)
        accs.append((a, tri))
    rays = np.concatenate([scenes.camera_rays(256, 256, seed=5), scenes.random_rays(60_000, seed=6)], axis=1)
    pool = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    return accs, pool


def make_batches(accs, pool, seed=0):
    from sort_b200 import Batch
    rng = np.random.default_rng(seed)
    sizes = [0, 1, 31, 1000, 4096, 17, 60_000, 5, 125_536, 2048, 333, 70_000]
    out = []
    for k, m in enumerate(sizes):
        acc = accs[k % len(accs)][0]
        a = int(rng.integers(0, pool.shape[1] - m + 1))
        out.append(Batch(acc, pool[:, a:a + m], any=bool(k % 3 == 2)))
    return out


def reference(batch):
    r = batch.rays.contiguous()
    if batch.any:
        return batch.accel.GetAttenuation(r)
    return batch.accel.GetIntersect(r)


def assert_same(batch):
    ref = reference(batch)
    torch.cuda.synchronize()
    if batch.any:
        assert torch.equal(ref, batch.occluded)
        return
    assert torch.equal(ref.prim, batch.hits.prim)
    for a, b in ((ref.t, batch.hits.t), (ref.u, batch.hits.u), (ref.v, batch.hits.v)):
        assert same_bits(a.cpu().numpy(), b.cpu().numpy())


def test_batches_match_single_scene_queries(world):
    from sort_b200 import Batcher
    accs, pool = world
    b = Batcher()
    batches = make_batches(accs, pool)
    b.run(batches)
    done = b.wait()
    assert not b.budget_cut
    assert np.all(done >= 0) and done[0] == 0
    for x in batches:
        assert_same(x)


def test_fp32_batches_match_sort(world, port):
    from sort_b200 import Batch, Batcher
    accs, pool = world
    b = Batcher()
    batches = [Batch(accs[0][0], pool[:, 100:30_100]), Batch(accs[1][0], pool[:, 7:50_007]),
               Batch(accs[1][0], pool[:, 0:20_000], any=True)]
    b.run(batches)
    b.wait()
    for x, (acc, tri) in zip(batches, [accs[0], accs[1], accs[1]]):
        tree = port.build(tri, acc.WIDTH)
        r = x.rays.cpu().numpy()
        if x.any:
            assert np.array_equal(tree.any(r), x.occluded.cpu().numpy())
        else:
            prim, t, _, _ = tree.closest(r)
            assert np.array_equal(prim, x.hits.prim.cpu().numpy())
            assert same_bits(t, x.hits.t.cpu().numpy())


@pytest.mark.parametrize("tuning", [{"block_threads": 64, "refill_threshold": 1},
                                    {"block_threads": 256, "refill_threshold": 32, "stack": 256},
                                    {"block_threads": 128, "refill_threshold": 8, "blocks_per_sm": 1}])
def test_results_independent_of_tuning_and_order(world, tuning):
    from sort_b200 import Batcher
    accs, pool = world
    b = Batcher()
    b.tuning = tuning
    batches = make_batches(accs, pool, seed=3)[::-1]
    b.run(batches)
    b.wait()
    for x in batches:
        assert_same(x)


def test_repeated_runs_reuse_tables(world):
    from sort_b200 import Batcher
    accs, pool = world
    b = Batcher(max_batches=16)
    for seed in range(6):  # more runs than staging buffers, enqueued back to back
        batches = make_batches(accs, pool, seed=seed)
        b.run(batches)
    b.wait()
    for x in batches:
        assert_same(x)


def test_time_budget_cuts_and_recovers(world):
    from sort_b200 import Batcher
    accs, pool = world
    b = Batcher()
    batches = make_batches(accs, pool, seed=1)
    b.run(batches, budget_ns=1)
    done = b.wait()
    assert b.budget_cut
    assert np.any(done < 0)
    b.run(batches)
    done = b.wait()
    assert not b.budget_cut and np.all(done >= 0)
    for x in batches:
        assert_same(x)


def test_autotune_picks_width_and_keeps_results(world, tmp_path):
    from sort_b200 import Batch, Batcher, Obvh, Qbvh
    accs, pool = world
    acc8, tri8 = accs[0]
    acc4, tri4 = accs[1]
    alt8 = Qbvh()
    alt8.Build(tri8)
    alt4 = Obvh()
    alt4.Build(tri4)
    batches = [Batch(acc8, pool[:, 0:40_000]), Batch(acc4, pool[:, 5_000:65_000]),
               Batch(acc8, pool[:, 1_000:9_000], any=True)]
    b = Batcher()
    cache = str(tmp_path / "tune.json")
    tuning, use = b.autotune(batches, [alt8, alt4, alt8], reps=2, cache=cache)
    assert tuning["block_threads"] in (64, 128, 256) and 1 <= tuning["refill_threshold"] <= 32
    assert use[0] == use[2]
    chosen = [Batch(alt8 if use[0] else acc8, batches[0].rays), Batch(alt4 if use[1] else acc4, batches[1].rays),
              Batch(alt8 if use[2] else acc8, batches[2].rays, any=True)]
    b.run(chosen)
    b.wait()
    for x in chosen:
        assert_same(x)
    b2 = Batcher()
    tuning2, use2 = b2.autotune(batches, [alt8, alt4, alt8], cache=cache)  # served from the cache
    assert tuning2 == tuning and use2 == use


def test_bad_arguments(world):
    from sort_b200 import Batch, Batcher, SortGpuError
    accs, pool = world
    b = Batcher(max_batches=2)
    with pytest.raises(SortGpuError, match="LIMIT"):
        b.run([Batch(accs[0][0], pool[:, :10])] * 3)
    with pytest.raises(SortGpuError, match="INVALID_ARGUMENT"):
        b.tuning = {"block_threads": 96}
