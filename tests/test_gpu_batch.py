"""Batched uneven chains (askja_batch_*): every chain of a mixed batch must
follow exactly the trajectory the same chain follows alone in the
single-chain engine (same links, seed, BETA, DT, LEVEL): the batched kernels
run the same per-link code, only the work distribution differs (FP32 chains
with NC <= 4 in the residual-plane mode, as a single FP32 chain)."""
import numpy as np
import pytest

import askja_b200 as ab

pytestmark = pytest.mark.gpu

CHAINS = [
    dict(nc=2, dims=[16, 16], beta=2.0, dt=0.05, level=8, seed=11),
    dict(nc=3, dims=[4, 8, 8, 8], beta=5.5, dt=0.02, level=6, seed=12),
    dict(nc=4, dims=[6, 6, 6], beta=9.0, dt=0.02, level=8, seed=13),
    dict(nc=8, dims=[4, 4, 4, 4], beta=40.0, dt=0.01, level=8, seed=14),
    dict(nc=3, dims=[5, 5, 5], beta=4.0, dt=0.03, level=7, seed=15),
    dict(nc=2, dims=[3, 16, 16, 4], beta=2.5, dt=0.04, level=5, seed=16),
]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_matches_single_chains(precision):
    nsteps, ntraj = 6, 3
    with ab.Batch(CHAINS, precision=precision) as b:
        b.hot_start(99)
        starts = [b.get_links(c) for c in range(len(CHAINS))]
        res = b.run(ntraj, nsteps, use_graph=True)
        ends = [b.get_links(c) for c in range(len(CHAINS))]
        plaq = b.plaquette()
    for c, ch in enumerate(CHAINS):
        with ab.Engine(ch["nc"], ch["dims"], beta=ch["beta"], dt=ch["dt"], level=ch["level"], precision=precision,
                       seed=ch["seed"]) as e:
            e.set_links(starts[c])
            last, _ = e.run_trajectories(ntraj, nsteps, use_graph=True)
            assert res[c]["n_tot"] == ntraj
            for k in ("h_old", "h_new", "dh", "u", "accepted", "n_acc", "n_rej"):
                assert res[c][k] == last[k], (c, k, res[c][k], last[k])
            np.testing.assert_array_equal(ends[c], e.get_links())
            vol = int(np.prod(ch["dims"]))
            nplaq = vol * len(ch["dims"]) * (len(ch["dims"]) - 1) / 2
            assert plaq[c] == pytest.approx(1.0 - e.EnergyMag() / nplaq, rel=1e-14)


def test_batch_graph_equals_eager():
    out = []
    for use_graph in (False, True):
        with ab.Batch(CHAINS[:4], precision="fp32") as b:
            b.hot_start(5)
            r = b.run(2, 5, use_graph=use_graph)
            out.append((r, [b.get_links(c) for c in range(4)]))
    assert out[0][0] == out[1][0]
    for a, c in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, c)


def test_batch_rejects_bad_chain():
    with pytest.raises(ab.AskjaError):
        ab.Batch([dict(nc=1, dims=[4, 4], beta=1.0, dt=0.1)])
    with ab.Batch(CHAINS[:1]) as b:
        with pytest.raises(ab.AskjaError):
            b.get_links(3)
        bad = b.get_links(0)
        bad[0, 0, 0, 0] = np.nan
        with pytest.raises(ab.AskjaError):
            b.set_links(0, bad)
