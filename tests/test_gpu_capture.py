"""Steps replayed from a captured CUDA graph (ogx_set_tuning with capture_steps = 1).

A captured step reads no counts back in the middle of its evaluation: its launches and
buffers are sized from capacities (the counts of the last eager evaluation plus an eighth),
every kernel takes its bounds from the counts on the device, and a step whose tree or
lists do not fit is redone eagerly inside the same ogx_step call.  Whichever way a step
goes, its result is the eager step's: positions, velocities and accelerations must be
bit-identical to the same steps taken eagerly (the leapfrog of VelocityVerlet3D::step,
src3d/Integrator3D.hpp:23-40).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(ogx, prec, pos, vel, mass, dt, steps, capture, p=6, thr=32):
    with ogx.AdaptiveFMM3D(p=p, threshold=thr, precision=prec) as s:
        if capture:
            s.set_tuning(capture_steps=1)
        s.upload(pos, vel, mass)
        for _ in range(steps):
            s.step(dt, 1)
        out = s.download()
        st = s.stats()
    return out, st


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_captured_steps_match_eager_steps_bit_for_bit(ogx, prec):
    import ogx_ic
    pos, vel, mass = ogx_ic.plummer(30000, seed=4)
    code = ogx.PREC_FP64 if prec == "fp64" else ogx.PREC_MIXED
    eager, st_e = _run(ogx, code, pos, vel, mass, 0.01, 7, capture=False)
    graph, st_g = _run(ogx, code, pos, vel, mass, 0.01, 7, capture=True)
    # step 1 sizes the buffers uncaptured, step 2 is recorded, steps 2..7 run from the graph
    assert st_g["graph_steps"] >= 5 and st_e["graph_steps"] == 0
    for a, b in zip(eager, graph):
        np.testing.assert_array_equal(a, b)


def test_a_step_that_outgrows_its_capacities_is_redone_eagerly(ogx):
    """Half of a Plummer sphere collapses twentyfold in one step: the tree gains levels
    and boxes beyond the capacities of the step before, the step is redone eagerly, and
    the run still equals the eager run bit for bit."""
    import ogx_ic
    pos, _, mass = ogx_ic.plummer(20000, seed=6)
    dt = 0.1
    vel = np.zeros_like(pos)
    half = pos[:, 0] > 0
    c = pos[half].mean(axis=0)
    vel[half] = (c - pos[half]) * (0.95 / dt)
    eager, _ = _run(ogx, ogx.PREC_MIXED, pos, vel, mass, dt, 4, capture=False)
    graph, st = _run(ogx, ogx.PREC_MIXED, pos, vel, mass, dt, 4, capture=True)
    assert st["step_redos"] >= 1
    for a, b in zip(eager, graph):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_captured_host_buffer_evaluations_match_eager_ones(ogx, prec):
    """ogx_eval on page-locked buffers with capture on: call 1 eager (sets the capacities),
    call 2 in capacity mode, call 3 recorded and replayed, later calls replayed; new contents
    in the same buffers that outgrow the capacities are redone eagerly; other buffers start
    over.  Every result equals the eager handle's bit for bit."""
    import torch
    import ogx_ic
    code = ogx.PREC_FP64 if prec == "fp64" else ogx.PREC_MIXED
    pos, _, mass = ogx_ic.plummer(30000, seed=9)
    n = pos.shape[0]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    pos_h, mass_h = pin(pos), pin(mass)
    acc_h = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
    # half of the bodies pulled twentyfold towards their centre: a deeper tree with more
    # boxes than the capacities of the first bodies allow
    pos2 = pos.copy()
    half = pos[:, 0] > 0
    c = pos[half].mean(axis=0)
    pos2[half] = c + (pos[half] - c) * 0.05

    def call(s, p_h, m_h, a_h):
        s.compute_accelerations_host_ptr(n, p_h.data_ptr(), m_h.data_ptr(), a_h.data_ptr())
        return a_h.numpy().copy()

    stream = torch.cuda.Stream()
    with ogx.AdaptiveFMM3D(p=6, threshold=32, precision=code) as e:
        ref1 = e.compute_accelerations(pos, mass)
        ref2 = e.compute_accelerations(pos2, mass)
    with ogx.AdaptiveFMM3D(p=6, threshold=32, precision=code, stream=stream.cuda_stream) as s:
        s.set_tuning(capture_steps=1)
        for _ in range(5):
            np.testing.assert_array_equal(call(s, pos_h, mass_h, acc_h), ref1)
        assert s.stats()["graph_evals"] == 3
        pos_h.copy_(torch.from_numpy(pos2))
        np.testing.assert_array_equal(call(s, pos_h, mass_h, acc_h), ref2)
        assert s.stats()["step_redos"] >= 1
        acc2_h = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
        for _ in range(3):
            np.testing.assert_array_equal(call(s, pos_h, mass_h, acc2_h), ref2)
