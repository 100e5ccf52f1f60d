"""Asynchronous state snapshots (nf_snapshot_begin / nf_snapshot_wait) on the GPU: a snapshot taken
between steps holds exactly the state of that moment although later steps were queued before the
wait, and the solver's own trajectory is unchanged by it."""
import numpy as np
import pytest

from helpers import config_for, golden, mesh
from netflux_b200 import _lib as L
from netflux_b200 import solver as S

pytestmark = pytest.mark.gpu


def test_snapshot_holds_the_state_of_its_moment():
    import torch
    g = golden("bump12")
    cfg = config_for(precision="fp64", freestream=tuple(g["freestream"]))
    a = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    a.advance(3)
    ref3 = a.get_solver_data().get_solution()
    a.advance(4)
    ref7 = a.get_solver_data().get_solution()
    a.close()

    b = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    b.advance(3)
    pinned = torch.empty((b.n_cells, 5), dtype=torch.float64, pin_memory=True).numpy()
    b.snapshot_begin(pinned)
    b.advance(4)  # queued after the snapshot, before the wait
    assert b.snapshot_wait() is pinned
    assert np.array_equal(pinned, ref3)
    assert np.array_equal(b.get_solver_data().get_solution(), ref7)

    pageable = np.empty((b.n_cells, 5))
    b.snapshot_begin(pageable)
    assert np.array_equal(b.snapshot_wait(), ref7)
    assert b.snapshot_wait() is None  # nothing in flight

    with pytest.raises(ValueError):
        b.snapshot_begin(np.empty((b.n_cells + 1, 5)))
    assert L.load().nf_snapshot_begin(b._h, L.dptr(pageable), b.n_cells + 1) == L.NF_ERR_ARG

    b.snapshot_begin(pinned)
    b.snapshot_begin(pageable)  # both in flight at once (two staging buffers), no host wait
    b.advance(2)
    assert np.array_equal(b.snapshot_wait(), ref7)
    b.snapshot_begin(pinned)
    b.close()  # destroying the solver waits for the copy in flight


def test_upload_commit_equals_set_state_and_streams_with_snapshots():
    """nf_upload_begin / nf_upload_commit: a state uploaded while other steps are queued becomes the
    solver's state exactly as set_state makes it; uploads and snapshots then stream independent
    states through one solver, both copies overlapping the steps."""
    import torch
    g = golden("bump12")
    cfg = config_for(precision="fp64", freestream=tuple(g["freestream"]))
    a = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    a.advance(2)
    Ua = a.get_solver_data().get_solution()
    a.set_state(Ua)
    a.advance(1)
    s1 = a.get_solver_data().get_solution()
    a.advance(2)
    s3 = a.get_solver_data().get_solution()
    a.close()

    def pinned(x):
        t = torch.empty(x.shape, dtype=torch.float64, pin_memory=True).numpy()
        t[:] = x
        return t

    ins = [pinned(Ua), pinned(Ua)]
    b = S.EulerSolver(cfg, mesh(g), U0=g["U0"])
    b.advance(1)
    b.upload_begin(ins[0])
    b.advance(2)  # queued on the old state while the copy runs
    b.upload_commit()
    b.advance(3)
    assert np.array_equal(b.get_solver_data().get_solution(), s3)

    with pytest.raises(L.NetFluxError):
        b.upload_commit()  # nothing in flight
    b.upload_begin(ins[0])
    with pytest.raises(L.NetFluxError):
        b.upload_begin(ins[1])  # one upload at a time
    b.upload_commit()
    assert np.array_equal(b.get_solver_data().get_solution(), Ua)
    with pytest.raises(ValueError):
        b.upload_begin(np.empty((b.n_cells, 4)))

    outs = [pinned(np.zeros_like(Ua)), pinned(np.zeros_like(Ua))]
    b.upload_begin(ins[0])
    for i in range(4):
        b.upload_commit()
        if i < 3:
            b.upload_begin(ins[(i + 1) % 2])  # the next state's copy overlaps this step
        b.advance(1)
        b.snapshot_begin(outs[i % 2])  # this result's copy overlaps the next upload and step
    b.snapshot_wait()
    b.upload_wait()  # the last input's copy has landed; its host buffer is free
    assert np.array_equal(outs[0], s1) and np.array_equal(outs[1], s1)
    b.upload_begin(ins[0])
    b.close()  # destroying the solver waits for the upload in flight
