"""Batched multiplication: one persistent launch over a global work queue,
graph-replayed, autotuned launch shape; every instance checked against the
oracle."""
import numpy as np
import pytest

import oracle
from lamb_b200.gen import WaterGeometry, batch_instances
from tests.helpers import assert_same_pattern, block_values, rel_frobenius_error

pytestmark = pytest.mark.gpu


def test_batch_of_uneven_instances(gpu_ctx):
    wls = batch_instances(n=6, seed=5, mol_range=(12, 80), cut_range=(4.0, 7.0))
    hosts, devs = [], []
    for i, wl in enumerate(wls):
        g, a, b = wl.build()
        da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
        if i % 2 == 0:
            da.set_positions(g.sector_positions(), g.box)
        dc = gpu_ctx.create_like(da)
        hosts.append((a, b, wl.eps))
        devs.append((da, db, dc))
    batch = gpu_ctx.batch([d[0] for d in devs], [d[1] for d in devs], [d[2] for d in devs], eps=1e-10)
    cfg = batch.config()
    assert cfg["warps"] in (4, 8) and cfg["cap"] in (16, 32) and cfg["grab"] in (1, 4, 16)
    assert cfg["order"] in ("instance", "shape")
    total = 0.0
    for rep in range(2):  # first execute captures the graph, the second replays it
        st = batch.execute()
        assert st["kernel_launches"] == 1
        for (a, b, eps), (_, _, dc) in zip(hosts, devs):
            c_ref, st_ref = oracle.multiply(a, b, eps, oracle.NO_RESULT_FILTER)
            c = dc.download()
            assert_same_pattern(c, c_ref)
            assert rel_frobenius_error(c, c_ref) <= 1e-12
            total += st_ref["flops"] if rep == 0 else 0.0
    assert abs(st["flops"] - total) <= 1e-6 * total
    batch.destroy()


def _no_borderline(c_ref, eps):
    for v in block_values(c_ref).values():
        assert abs(float(np.sqrt(np.sum(v ** 2))) - eps) > 1e-9 * eps


def test_batch_full_run_with_filters(gpu_ctx):
    """lamb_gpu_batch_run(FULL): symbolic phase, graph-replayed numeric launch
    and result filter of every instance, O 23 and O 13 instances, both
    filters active; every C against the oracle with the same filters, twice
    (the second full run refreshes the queue in place and replays)."""
    eps = 3e-2  # drops products and C blocks in these boxes
    wls = batch_instances(n=4, seed=7, mol_range=(16, 60), cut_range=(4.5, 7.0))
    assert {wl.blk_o for wl in wls} == {13, 23}
    hosts, devs = [], []
    for wl in wls:
        g, a, b = wl.build()
        da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
        da.set_positions(g.sector_positions(), g.box)
        hosts.append((a, b))
        devs.append((da, db, gpu_ctx.create_like(da)))
    batch = gpu_ctx.batch([d[0] for d in devs], [d[1] for d in devs], [d[2] for d in devs], eps=eps)
    refs = [oracle.multiply(a, b, eps) for a, b in hosts]
    for c_ref, _ in refs:
        _no_borderline(c_ref, eps)
    assert sum(st["n_products_skipped"] for _, st in refs) > 0
    assert sum(st["n_c_blocks_dropped"] for _, st in refs) > 0
    for rep in range(2):
        st = batch.run_full()
        assert st["ms_symbolic"] > 0 and st["ms_numeric"] > 0 and st["ms_total"] >= st["ms_numeric"]
        assert st["n_c_blocks_dropped"] == sum(r[1]["n_c_blocks_dropped"] for r in refs)
        assert st["n_products"] == sum(r[1]["n_products"] for r in refs)
        for (c_ref, _), (_, _, dc) in zip(refs, devs):
            c = dc.download()
            assert_same_pattern(c, c_ref)
            assert rel_frobenius_error(c, c_ref) <= 1e-12
        assert st["n_c_blocks"] == sum(sum(s.n_blks for s in r[0].sectors) for r in refs)
    batch.destroy()


def test_batch_refuses_changed_operands(gpu_ctx):
    """The graph holds the operands' device pointers: once C is re-multiplied
    (new layout) or an operand is destroyed, execute returns lamb_wrong_args
    before launching anything."""
    from lamb_b200.gpu import LambError
    g = WaterGeometry(16, None, 5.0, seed=2)
    a, b = g.matrix(1), g.matrix(2)
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    dc = gpu_ctx.create_like(da)
    batch = gpu_ctx.batch([da], [db], [dc], eps=1e-10)
    batch.execute()
    gpu_ctx.multiply(da, db, dc, 1e-10)       # replaces C's buffers
    with pytest.raises(LambError) as e:
        batch.execute()
    assert e.value.type == 100
    batch.destroy()
    batch = gpu_ctx.batch([da], [db], [dc], eps=1e-10)
    db.destroy()
    with pytest.raises(LambError) as e:
        batch.execute()
    assert e.value.type == 100
    batch.destroy()
    dc.destroy()
    da.destroy()


def test_batch_rejects_shared_outputs(gpu_ctx):
    g = WaterGeometry(16, None, 5.0, seed=1)
    a = g.matrix(1)
    da = gpu_ctx.upload(a)
    dc = gpu_ctx.create_like(da)
    from lamb_b200.gpu import LambError
    with pytest.raises(LambError):
        gpu_ctx.batch([da, da], [da, da], [dc, dc])
