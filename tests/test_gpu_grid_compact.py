"""GPU gridding and compaction against the oracle: bit-exact counts, scaled
masses, cell indices and compaction order."""
import numpy as np
import pytest

from flexpart_gpu.records import PARTICLE_DTYPE
from helpers import population
from oracle import orc

pytestmark = pytest.mark.gpu

api = pytest.importorskip("flexpart_gpu.api")


@pytest.fixture(scope="module")
def ctx():
    c = api.Context(0)
    yield c
    c.close()


def test_gridding_reference_case(ctx):
    # tests/integration/scientific_invariants.rs:93-164
    pts = [(2, 3, 50.0, 1.5), (2, 3, 150.0, 0.8), (5, 1, 600.0, 2.0), (7, 5, 999.0, 0.3), (0, 0, 10.0, 4.0),
           (1, 1, 80.0, 9.9)]
    rec = np.zeros(len(pts), PARTICLE_DTYPE)
    for i, (cx, cy, z, m) in enumerate(pts):
        rec[i]["cell_x"], rec[i]["cell_y"], rec[i]["pos_x"], rec[i]["pos_y"], rec[i]["pos_z"] = cx, cy, 0.3, 0.6, z
        rec[i]["mass"][0] = m
        rec[i]["flags"] = 0 if i == 5 else 1
    p = api.Particles(ctx, len(pts))
    p.upload(rec)
    g = api.Grid(ctx, 8, 6, 3)
    g.accumulate(p, 0, 1e6, [100.0, 500.0, 1000.0])
    counts, mass, kg = g.download()
    oc, om, _ = orc.grid(orc.State.from_records(rec), len(pts), 0, 1e6, [100.0, 500.0, 1000.0], (8, 6, 3))
    assert np.array_equal(counts, oc) and np.array_equal(mass, om)
    assert counts.sum() == 5
    assert np.array_equal(kg, (om.astype(np.float32) / np.float32(1e6)).astype(np.float32))


@pytest.mark.parametrize("outheights", [[100.0, 500.0, 1000.0], [0.0, 0.0, 0.0, 0.0],
                                        [500.0, 100.0, 1000.0],                      # unsorted: the scan
                                        [50.0 * (k + 1) for k in range(12)],         # sorted, beyond the count
                                        [100.0, 100.0, 400.0, 400.0, 800.0, 1600.0, 3200.0, 6400.0]])
def test_gridding_bit_exact_large(ctx, outheights):
    nx, ny = 40, 30
    rec = population(nx, ny, 200_003, seed=3, z_max=2000.0 if outheights[0] > 0 else 5.0)
    rec["cell_x"][::11] = -3            # out-of-range cells are clamped
    rec["cell_y"][::13] = ny + 5
    rec["mass"][::17, 0] = -1.0          # negative mass counts, adds 0
    rec["mass"][::19, 0] = 5000.0        # saturates the u32 quantisation
    p = api.Particles(ctx, len(rec))
    p.upload(rec)
    nz = len(outheights)
    g = api.Grid(ctx, nx, ny, nz)
    g.accumulate(p, 0, 1e6, outheights)
    counts, mass, _ = g.download()
    st = orc.State.from_records(rec)
    oc, om, ocell = orc.grid(st, len(rec), 0, 1e6, outheights, (nx, ny, nz))
    assert np.array_equal(counts, oc)
    assert np.array_equal(mass, om)
    assert np.array_equal(g.cell_indices(p, outheights), ocell)
    # deterministic: a second pass gives the same bits
    g.accumulate(p, 0, 1e6, outheights)
    c2, m2, _ = g.download()
    assert np.array_equal(c2, counts) and np.array_equal(m2, mass)


@pytest.mark.parametrize(
    "n,inactive",
    [(1000, lambda i: i % 3 == 0), (512, lambda i: False), (256, lambda i: True), (100, lambda i: i != 42),
     (300, lambda i: i % 5 == 0), (1000, lambda i: i % 2 == 0), (70_001, lambda i: (i * 2654435761) % 7 < 3)],
)
def test_compaction_matches_reference_sets_and_order(ctx, n, inactive):
    # src/gpu/compaction.rs:624-740 plus order and the deactivated tail
    rec = population(50, 50, n, seed=n, inactive_every=0)
    rec["flags"] = np.array([0 if inactive(i) else 1 for i in range(n)], np.uint32)
    rec["time"] = np.arange(n, dtype=np.int32)
    p = api.Particles(ctx, n)
    p.upload(rec)
    comp = api.Compaction(ctx, n)
    idx = api.DeviceArray(ctx, n, np.uint32)
    count = comp.compact(p, idx)
    out_ref, count_ref, idx_ref = orc.compact_records(rec)
    assert count == count_ref
    assert p.dispatch_count == count_ref
    assert np.array_equal(idx.numpy()[:count], idx_ref)
    assert np.array_equal(p.download(), out_ref)


@pytest.mark.parametrize("n,heights", [(100_003, True), (4_097, False)])
def test_sort_by_cell_matches_oracle_permutation(ctx, n, heights):
    from helpers import production_params, small_met
    spec, frames, met = small_met(nz=16, heights=heights)
    rec = population(spec.nx, spec.ny, n, seed=5, z_max=3000.0 if heights else 15.0)
    rec["time"] = np.arange(n, dtype=np.int32)
    p = api.Particles(ctx, n)
    p.upload(rec)
    m = api.Met(ctx, spec.nx, spec.ny, spec.nz)
    m.upload_frame(0, met["u0"], met["v0"], met["w0"])
    m.upload_frame(1, met["u1"], met["v1"], met["w1"])
    m.set_level_heights(met["heights"])
    srt = api.Sorter(ctx, n)
    perm = api.DeviceArray(ctx, n, np.uint32)
    srt.sort(p, m, perm)
    ref, ref_perm = orc.sort_by_cell(rec, n, met["heights"], (spec.nx, spec.ny, spec.nz))
    assert np.array_equal(perm.numpy(), ref_perm)
    assert np.array_equal(p.download(), ref)
    # a partial dispatch range leaves the tail in place
    p.upload(rec)
    p.dispatch_count = n // 2
    srt.sort(p, m)
    ref2, _ = orc.sort_by_cell(rec, n // 2, met["heights"], (spec.nx, spec.ny, spec.nz))
    assert np.array_equal(p.download(), ref2)


def test_async_grid_download_orders_against_the_next_accumulate(ctx):
    """fpg_grid_download_async on a side stream into page-locked memory: the
    copy sees the grid of the accumulate before it, and the next accumulate
    into the same grid does not overwrite it before the copy is done."""
    import ctypes

    import torch

    nx, ny = 40, 30
    oh = [100.0, 500.0, 1000.0]
    ra = population(nx, ny, 300_000, seed=5, z_max=2000.0)
    rb = population(nx, ny, 300_000, seed=6, z_max=2000.0)
    pa, pb = api.Particles(ctx, len(ra)), api.Particles(ctx, len(rb))
    pa.upload(ra)
    pb.upload(rb)
    g = api.Grid(ctx, nx, ny, 3)
    cells = nx * ny * 3
    side = torch.cuda.Stream()
    bufs = [torch.zeros(cells, dtype=torch.int32, pin_memory=True) for _ in range(4)]
    g.accumulate(pa, 0, 1e6, oh)
    g.download_async(bufs[0].data_ptr(), bufs[1].data_ptr(), ctypes.c_void_p(side.cuda_stream))
    g.accumulate(pb, 0, 1e6, oh)
    g.download_async(bufs[2].data_ptr(), bufs[3].data_ptr(), ctypes.c_void_p(side.cuda_stream))
    side.synchronize()
    ctx.synchronize()
    for rec, c, m in ((ra, bufs[0], bufs[1]), (rb, bufs[2], bufs[3])):
        oc, om, _ = orc.grid(orc.State.from_records(rec), len(rec), 0, 1e6, oh, (nx, ny, 3))
        assert np.array_equal(c.numpy().view(np.uint32), oc)
        assert np.array_equal(m.numpy().view(np.uint32), om)
