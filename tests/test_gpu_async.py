"""Asynchronous host interface: askja_set_links_async (copy stream, two device
staging buffers used in turn) and askja_trajectory_async (graph replay, outcome
copied to pinned host memory).  A pipelined sequence of uploads and
trajectories must give exactly what the synchronous calls give."""
import ctypes

import numpy as np
import pytest

import askja_b200 as ab
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu


def configs(nc, dims, k, seed):
    rng = np.random.default_rng(seed)
    O = Oracle(nc, dims)
    return [fields.haar(nc, O.vol * O.dim, rng).reshape(O.shape) for _ in range(k)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_upload_matches_set_links(precision):
    nc, dims = 3, [4, 4, 2, 4]
    (u,) = configs(nc, dims, 1, 4)
    buf = ab.PinnedBuffer.alloc(u.nbytes)
    try:
        buf.array(np.complex128, u.shape)[...] = u
        with ab.Engine(nc, dims, beta=5.7, precision=precision) as e:
            e.set_links_async(buf.ptr)
            e.sync()
            got, saved = e.get_links(), e.get_saved_links()
            e.set_links(u)
            want = e.get_links()
        assert np.array_equal(got, want)
        assert np.array_equal(saved, want)
    finally:
        buf.free()


@pytest.mark.parametrize("nc,dims,precision", [(3, [4, 4, 4, 4], "fp32"), (3, [4, 3, 4], "fp64"),
                                               (8, [3, 4, 2], "fp32"), (32, [2, 2, 2], "fp32")])
def test_pipeline_matches_synchronous_calls(nc, dims, precision):
    """Five configurations through two host buffers: upload k+1 is enqueued
    while trajectory k runs; each trajectory's outcome and the final links
    equal those of set_links + trajectory."""
    us = configs(nc, dims, 5, 17 + nc)
    nsteps = 6
    with ab.Engine(nc, dims, beta=2.0 * nc, dt=0.02, precision=precision, seed=5) as e:
        want = []
        for u in us:
            e.set_links(u)
            want.append(e.trajectory(nsteps))
        want_links = e.get_links()
    bufs = [ab.PinnedBuffer.alloc(us[0].nbytes) for _ in range(2)]
    rsz = ctypes.sizeof(ab.TrajResult)
    res = ab.PinnedBuffer.alloc(rsz * len(us))
    try:
        with ab.Engine(nc, dims, beta=2.0 * nc, dt=0.02, precision=precision, seed=5) as e:
            for k, u in enumerate(us):
                if k >= 2:
                    e.sync()  # host buffer k % 2 is refilled only after its copy has run
                bufs[k % 2].array(np.complex128, u.shape)[...] = u
                e.set_links_async(bufs[k % 2].ptr)
                e.trajectory_async(nsteps, res.ptr + k * rsz)
            e.sync()
            got = [ab.TrajResult.from_address(res.ptr + k * rsz).as_dict() for k in range(len(us))]
            got_links = e.get_links()
    finally:
        for b in bufs:
            b.free()
        res.free()
    for g, w in zip(got, want):
        assert g == w
    assert np.array_equal(got_links, want_links)


def test_nonfinite_upload_reported_at_sync():
    nc, dims = 3, [4, 4]
    (u,) = configs(nc, dims, 1, 9)
    u = u.copy()
    u[3, 1, 0, 2] = np.nan
    buf = ab.PinnedBuffer.alloc(u.nbytes)
    try:
        buf.array(np.complex128, u.shape)[...] = u
        with ab.Engine(nc, dims, beta=5.7) as e:
            e.set_links_async(buf.ptr)
            with pytest.raises(ab.AskjaError) as ei:
                e.sync()
            assert "non-finite" in str(ei.value)
            e.sync()  # reported once
            e.initializeU()
            assert np.isfinite(e.trajectory(4)["dh"])
    finally:
        buf.free()
