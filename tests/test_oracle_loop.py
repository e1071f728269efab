"""The oracle's restatement of the engine's impulse loop, on the CPU."""
import numpy as np


def test_loop_reduces_contacts_and_stops(oracle):
    from cccollisions_b200 import workloads as W
    v0, v1, vel, faces, masses = W.impulse_fold_mesh(3, 14, 12)
    ev1, evel, it, conv, per = oracle.impulse_loop(v0, v1, vel, faces, masses, max_iter=50)
    assert per[0] > 0                       # the fold collides
    assert 1 <= it <= 50
    if conv:
        assert per[-1] == 0 and len(per) == it + 1
    # vertices that no contact touched keep their end positions
    moved = np.any(ev1 != v1, axis=1)
    assert moved.any() and not moved.all()


def test_loop_is_deterministic_and_respects_max_iter(oracle):
    from cccollisions_b200 import workloads as W
    v0, v1, vel, faces, masses = W.impulse_fold_mesh(5, 12, 12)
    a = oracle.impulse_loop(v0, v1, vel, faces, masses, max_iter=3, nthreads=1)
    b = oracle.impulse_loop(v0, v1, vel, faces, masses, max_iter=3, nthreads=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert a[2] <= 3


def test_collision_free_input_converges_at_once(oracle):
    from cccollisions_b200 import workloads as W
    v, f = W.grid(6, 6)
    v = v.astype(np.float64)
    v1 = v.copy()
    v1[:, 2] -= 0.01
    m = np.ones((f.shape[0], 3))
    ev1, evel, it, conv, per = oracle.impulse_loop(v, v1, v1 - v, f.astype(np.int32), m)
    assert it == 0 and conv and per.tolist() == [0]
    assert np.array_equal(ev1, v1)


def test_separated_fold_converges(oracle):
    """The fold whose layers start apart (workloads.SEPARATED_FOLD): every triangle collides in
    the first check, and the loop separates the layers within a few iterations."""
    from cccollisions_b200 import workloads as W
    v0, v1, vel, faces, masses = W.impulse_fold_mesh(7, 24, 20, **W.SEPARATED_FOLD)
    ev1, evel, it, conv, per = oracle.impulse_loop(v0, v1, vel, faces, masses, max_iter=50)
    assert conv and 1 <= it <= 5
    assert per[0] > faces.shape[0] and per[it] == 0
