"""Times every launch schedule of the resident engine on the batched CCD step and checks
each schedule's rows against the reference's digests in ``full_batched.npz``.

    python tests/golden/sweep_schedules.py [--meshes 64] [--only 4,10] [--steps 5]

One JSON line per schedule: the schedule's fields (traversal and narrow blocks an SM, warp
traversal), the meshes whose rows differ from the reference's (``bad``, empty when equal),
the work counters of the last step and the mean device time of each kernel over
``--steps`` steps.  Needs a CUDA device.
"""
import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch  # noqa: E402

from cccollisions_b200 import _native as N  # noqa: E402
from cccollisions_b200 import workloads as W  # noqa: E402
from cccollisions_b200.engine import Engine  # noqa: E402
from make_full_golden import row_digest  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--meshes", type=int, default=64)
    ap.add_argument("--only", default="", help="comma-separated schedule indices (default: all)")
    ap.add_argument("--steps", type=int, default=5)
    args = ap.parse_args()
    only = {int(x) for x in args.only.split(",") if x}
    digests = np.load(os.path.join(HERE, "full_batched.npz"))["digests"]
    meshes = W.batched()[:args.meshes]
    sizes = [a.shape[0] for a, _ in meshes]
    eng = Engine(tri_capacity=sum(sizes) + 64, mesh_capacity=64, max_candidates_per_triangle=32,
                 max_collisions_per_triangle=16)
    sids = [eng.add_mesh(f) for f in sizes]
    for sid, (a, b) in zip(sids, meshes):
        eng.upload_soup(sid, a, b)
    stream = torch.cuda.Stream()
    failed = False
    with torch.cuda.stream(stream):
        eng.set_active(sids)
        eng.build(sids)
        for i, sched in enumerate(Engine.schedules()):
            if only and i not in only:
                continue
            eng.set_schedule(i)
            eng.ccd()
            stream.synchronize()
            st = eng.state(sids)
            bad = []
            for k, sid in enumerate(sids):
                rows = eng.collisions(sid, int(st["rows"][k]))
                if row_digest(*[x.cpu().numpy() for x in rows]) != str(digests[k]):
                    bad.append(k)
            failed |= bool(bad)
            for _ in range(2):
                eng.ccd()
            N.timing_begin()
            for _ in range(args.steps):
                eng.ccd()
            kern = N.timing_end()
            stream.synchronize()
            print(json.dumps({"schedule": i, **sched, "bad": bad, "counters": eng.counters(),
                              "ms": {k: round(v[0] / v[1], 4) for k, v in kern.items()}}), flush=True)
    eng.close()
    sys.exit(1 if failed else 0)


if __name__ == "__main__":
    main()
