"""Frame readouts of every replica's stacks.  Overlapped dense readout
(edm_frame_out_begin / edm_frame_out_wait) and the sparse readout of the
nonzero bins (edm_frame_out_sparse): on two frames in a row, each equals the
stacks edm_get_flim returns replica by replica, and the live stacks start the
next frame cleared."""
import numpy as np
import pytest
import torch

from flim_microscopy_simulator_with_causal_inference_b200 import workloads as W
from flim_microscopy_simulator_with_causal_inference_b200.batch import Ensemble

pytestmark = pytest.mark.gpu


def test_frame_out_equals_per_replica_reads_on_two_frames():
    raws = W.ensemble_replicas(4, seed=11, n_min=600, n_max=1500)
    ens = Ensemble(raws, precision=32, photons=True, device=0)
    eng = ens.engine
    n = eng.flim_elems()
    sizes = [int(np.prod(eng.flim(r).shape)) for r in range(ens.R)]
    assert n == sum(sizes)
    host = torch.empty(n, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    s = torch.cuda.Stream()
    for frame in range(2):
        eng.pipeline_steps(50, True, 50, stream=s)
        eng.finalize(frame, stream=s)
        s.synchronize()
        expect = np.concatenate([eng.flim(r).ravel() for r in range(ens.R)])
        assert expect.sum() > 0
        host[:] = 7
        eng.frame_out_begin(host, stream=s)
        eng.frame_out_wait()
        np.testing.assert_array_equal(host, expect)
        s.synchronize()
        assert all(eng.flim(r).sum() == 0 for r in range(ens.R))


def test_frame_out_rejects_a_short_buffer():
    ens = Ensemble(W.ensemble_replicas(2, seed=3, n_min=600, n_max=800), precision=32, photons=True, device=0)
    short = np.zeros(ens.engine.flim_elems() - 1, dtype=np.uint32)
    with pytest.raises(RuntimeError, match="too small"):
        ens.engine.frame_out_begin(short)


def test_sparse_frame_out_equals_dense_stacks_on_two_frames():
    raws = W.ensemble_replicas(4, seed=11, n_min=600, n_max=1500)
    ens = Ensemble(raws, precision=32, photons=True, device=0)
    eng = ens.engine
    n = eng.flim_elems()
    cap = n // 16
    idx = np.full(cap, -1, dtype=np.int64)
    cnt = np.zeros(cap, dtype=np.uint32)
    s = torch.cuda.Stream()
    for frame in range(2):
        eng.pipeline_steps(50, True, 50, stream=s)
        eng.finalize(frame, stream=s)
        s.synchronize()
        expect = np.concatenate([eng.flim(r).ravel() for r in range(ens.R)])
        nnz = eng.frame_out_sparse(idx, cnt, stream=s)
        assert nnz == int(np.count_nonzero(expect)) > 0
        assert np.all(np.diff(idx[:nnz]) > 0)  # index order
        np.testing.assert_array_equal(eng.sparse_to_dense(idx, cnt, nnz, n), expect)
        assert all(eng.flim(r).sum() == 0 for r in range(ens.R))


def test_sparse_frame_out_beyond_capacity_leaves_the_stacks():
    ens = Ensemble(W.ensemble_replicas(2, seed=5, n_min=600, n_max=800), precision=32, photons=True, device=0)
    eng = ens.engine
    s = torch.cuda.Stream()
    eng.pipeline_steps(50, True, 50, stream=s)
    eng.finalize(0, stream=s)
    s.synchronize()
    before = np.concatenate([eng.flim(r).ravel() for r in range(ens.R)])
    assert np.count_nonzero(before) > 1
    idx = np.zeros(1, dtype=np.int64)
    cnt = np.zeros(1, dtype=np.uint32)
    with pytest.raises(RuntimeError, match="exceed the capacity"):
        eng.frame_out_sparse(idx, cnt, stream=s)
    after = np.concatenate([eng.flim(r).ravel() for r in range(ens.R)])
    np.testing.assert_array_equal(after, before)


def test_sparse_frame_out_sees_dark_counts_and_afterpulses():
    """Every writer of the stacks marks the stretches it touches: the
    detection pass, dark counts and afterpulsing (rich_small has both, at high
    rates), so the sparse read equals the dense stacks."""
    from tests import cases
    from tests.harness import Pair
    P = Pair(cases.get("rich_small"), precision=32, photons=True)
    eng = P.eng
    n = eng.flim_elems()
    idx = np.zeros(n, dtype=np.int64)
    cnt = np.zeros(n, dtype=np.uint32)
    s = torch.cuda.Stream()
    for frame in range(2):
        eng.pipeline_steps(30, True, 30, stream=s)
        eng.finalize(frame, stream=s)
        s.synchronize()
        expect = eng.flim(0).ravel().copy()
        c = eng.counters()[0]
        assert c[11] > 0 and c[12] > 0, "the system should produce dark counts and afterpulses"
        nnz = eng.frame_out_sparse(idx, cnt, stream=s)
        assert nnz == int(np.count_nonzero(expect)) > 0
        np.testing.assert_array_equal(eng.sparse_to_dense(idx, cnt, nnz, n), expect)
