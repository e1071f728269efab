"""Streamed collision steps (engine.StepPipeline) on the GPU.

Every step's packed rows, split back into meshes with the step's offsets, equal the rows of
the same step run alone through Engine.ccd() (as multisets, times bit for bit), for steps
whose inputs alternate between two motions of the same meshes.
"""
from collections import Counter

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ms(rows, times):
    return Counter(zip(map(tuple, np.asarray(rows).tolist()), np.asarray(times, dtype=np.float64).tolist()))


@pytest.mark.parametrize("graph", [True, False])
def test_pipeline_steps_equal_single_steps(cuda, graph):
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    from cccollisions_b200.engine import Engine, StepPipeline
    meshes = [W.jittered_fold(200 + i, nx, ny) for i, (nx, ny) in enumerate([(12, 9), (7, 15), (14, 14)])]
    other = [(x0, x0 + 0.6 * (x1 - x0)) for x0, x1, _ in meshes]        # a second motion of the same meshes
    eng = Engine(tri_capacity=sum(x0.shape[0] for x0, _, _ in meshes) + meshes[0][0].shape[0] + 20 + 32,
                 mesh_capacity=8)
    sids = [eng.add_mesh(x0.shape[0]) for x0, _, _ in meshes]
    # an inactive mesh between two active ones must keep its soups
    spare = eng.add_mesh(20)
    last = eng.add_mesh(meshes[0][0].shape[0])
    sids.append(last)
    sets = [[(x0, x1) for x0, x1, _ in meshes] + [(meshes[0][0], meshes[0][1])], other + [other[0]]]
    spare_x0 = np.random.default_rng(3).random((20, 3, 3))
    eng.upload_soup(spare, spare_x0, spare_x0)
    expect = []
    eng.set_active(sids)
    for k, soups in enumerate(sets):
        for sid, (a, b) in zip(sids, soups):
            eng.upload_soup(sid, a, b)
        if k == 0:
            eng.build(sids)
        eng.ccd()
        st = eng.state(sids)
        expect.append({sid: _ms(*[x.cpu().numpy() for x in eng.collisions(sid, int(n))])
                       for sid, n in zip(sids, st["rows"])})
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        if graph:
            eng.capture(N.ENGINE_OP_CCD)
    s.synchronize()
    pipe = StepPipeline(eng, sids, graph=graph)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    host = [[(pin(a), pin(b)) for a, b in soups] for soups in sets]
    order = [0, 1, 1, 0, 1]
    outs = [pipe.host_outputs() for _ in order]
    totals = pipe.run([host[i] for i in order], outs)
    M = len(sids)
    for k, i in enumerate(order):
        rows, times, meta = [o.numpy() for o in outs[k]]
        off, ids = meta[:M + 1], meta[M + 1:2 * M + 1]
        assert totals[k] == off[M] == sum(sum(c.values()) for c in expect[i].values())
        assert meta[2 * M + 1] == 0
        assert sorted(ids.tolist()) == sorted(sids)
        for m, sid in enumerate(ids.tolist()):
            got = _ms(rows[off[m]:off[m + 1]], times[off[m]:off[m + 1]])
            assert got == expect[i][sid], (k, sid)
    assert np.array_equal(eng.view(spare)["x0"].cpu().numpy(), spare_x0)
    # one output triple for every step: it ends up holding the last step
    one = pipe.host_outputs()
    totals = pipe.run([host[i] for i in order], [one] * len(order))
    rows, times, meta = [o.numpy() for o in one]
    off, ids = meta[:M + 1], meta[M + 1:2 * M + 1]
    assert off[M] == totals[-1]
    for m, sid in enumerate(ids.tolist()):
        assert _ms(rows[off[m]:off[m + 1]], times[off[m]:off[m + 1]]) == expect[order[-1]][sid]
    eng.close()


def test_pack_rows_capacity_and_meta(cuda):
    """pack_rows with room for fewer rows than the step produced: the first `capacity` rows
    are packed, the offsets still count every row, and the status word reports the overflow;
    with room for all rows each mesh's slice equals its own rows."""
    from cccollisions_b200 import _native as N
    from cccollisions_b200 import workloads as W
    from cccollisions_b200.engine import Engine
    meshes = [W.jittered_fold(220 + i, 12, 10) for i in range(3)]
    eng = Engine(tri_capacity=sum(x0.shape[0] for x0, _, _ in meshes) + 16, mesh_capacity=4)
    sids = [eng.add_mesh(x0.shape[0]) for x0, _, _ in meshes]
    for sid, (x0, x1, _) in zip(sids, meshes):
        eng.upload_soup(sid, x0, x1)
    eng.set_active(sids)
    eng.build(sids)
    eng.ccd()
    st = eng.state(sids)
    counts = dict(zip(sids, (int(n) for n in st["rows"])))
    total = sum(counts.values())
    assert total > 10
    M = len(sids)
    meta = torch.empty(2 * M + 2, dtype=torch.int32, device=cuda)
    rows = torch.full((total, 3), -7, dtype=torch.int64, device=cuda)
    times = torch.full((total,), -7.0, dtype=torch.float64, device=cuda)
    eng.pack_rows(rows, times, meta)
    m = meta.cpu().numpy()
    assert m[M] == total and m[2 * M + 1] == 0
    for i, sid in enumerate(m[M + 1:2 * M + 1].tolist()):
        r, t = eng.collisions(sid, counts[sid])
        assert m[i + 1] - m[i] == counts[sid]
        got = _ms(rows[m[i]:m[i + 1]].cpu().numpy(), times[m[i]:m[i + 1]].cpu().numpy())
        assert got == _ms(r.cpu().numpy(), t.cpu().numpy())
    small = total // 2
    rows2 = torch.full((small, 3), -7, dtype=torch.int64, device=cuda)
    times2 = torch.full((small,), -7.0, dtype=torch.float64, device=cuda)
    eng.pack_rows(rows2, times2, meta)
    assert int(meta[M]) == total
    assert (rows2 >= 0).all()
    assert eng.state([])["status"] & N.CCC_ST_OUT_OVERFLOW
    eng.close()
