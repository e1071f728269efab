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
    eng.close()
