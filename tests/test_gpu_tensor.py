"""Tensor-core link update (kernel_path 2: FP32 storage, NC = 16, 32 and 64,
every complex product a split-TF32 tcgen05 MMA; NC = 16 on the padded
M = 64 shape) against the FP64 oracle.

Tolerances are those of the FP32 CUDA-core path: the split keeps about 22
mantissa bits per operand and accumulates in FP32, so force and link errors
sit at FP32 rounding (relative 5e-5 on the kicked momenta, where the force is
a difference of nearly equal staple products, and 5e-6 on links)."""
import numpy as np
import pytest

import askja_b200 as ab
from conftest import rel
from oracle import Oracle, fields

pytestmark = pytest.mark.gpu

CASES = [(16, [2, 2, 2]), (16, [3, 2, 2]), (32, [2, 2, 2]), (32, [3, 2]), (64, [2, 2]), (64, [2, 3, 2])]
IDS = [f"su{n}_{'x'.join(map(str, d))}" for n, d in CASES]


def setup(nc, dims, seed):
    rng = np.random.default_rng(seed)
    O = Oracle(nc, dims)
    nl = O.vol * O.dim
    u = fields.haar(nc, nl, rng).reshape(O.shape)
    beta = 2.0 * nc * nc
    pi = fields.momenta(nc, nl, beta, rng, O)
    return O, u, pi, beta


def unitarity(u):
    m = u.reshape(-1, u.shape[-2], u.shape[-1])
    eye = np.eye(m.shape[-1])
    return float(np.max(np.abs(np.conj(np.swapaxes(m, -1, -2)) @ m - eye)))


@pytest.mark.parametrize("nc,dims", CASES, ids=IDS)
def test_kick_and_drift_vs_oracle(nc, dims):
    O, u, pi, beta = setup(nc, dims, nc + len(dims))
    with ab.Engine(nc, dims, beta=beta, dt=0.005, level=8, precision="fp32", reunitarise=False,
                   kernel_path=2) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.updateE(0.005)
        Pi = O.updateE(u, pi, 0.005)
        assert rel(e.get_momenta(1), Pi) < 5e-5
        # the force itself: (pi - Pi) / eps
        f_gpu = (pi - e.get_momenta(1)) / 0.005
        f_ref = (pi - Pi) / 0.005
        assert rel(f_gpu, f_ref) < 1e-4
        e.updateUandcopyDown(0.005)
        assert rel(e.get_links(), O.updateU(u, Pi, 0.005, 8)) < 5e-6


@pytest.mark.parametrize("nc,dims", CASES, ids=IDS)
@pytest.mark.parametrize("reunit", [False, True])
def test_leapfrog_vs_oracle(nc, dims, reunit):
    O, u, pi, beta = setup(nc, dims, 3 * nc + len(dims))
    with ab.Engine(nc, dims, beta=beta, dt=0.005, level=8, precision="fp32", reunitarise=reunit,
                   kernel_path=2) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.leapfrog(3, 0.005)
        uu, pp = u, O.updateE(u, pi, 0.0025)
        for k in range(3):
            uu = O.updateU(uu, pp, 0.005, 8)
            pp = O.updateE(uu, pp, 0.005 if k < 2 else 0.0025)
        got = e.get_links()
        assert rel(got, uu) < 1e-5
        assert rel(e.get_momenta(0), pp) < 5e-5
        if reunit:
            assert unitarity(got) < 2e-6


@pytest.mark.parametrize("order", [0, 1, 2, 8, 9])
def test_taylor_orders(order):
    """LEVEL 0 (exp = 1), 1 (no Horner product), 2, 8 and out-of-range (acts as 8)."""
    nc, dims = 32, [2, 2]
    O, u, pi, beta = setup(nc, dims, 11 + order)
    with ab.Engine(nc, dims, beta=beta, dt=0.01, level=order, precision="fp32", reunitarise=False,
                   kernel_path=2) as e:
        e.set_links(u)
        e.set_momenta(pi, 1)
        e.updateUandcopyDown(0.01)
        eff = order if 0 <= order <= 8 else 8
        assert rel(e.get_links(), O.updateU(u, pi, 0.01, eff)) < 5e-6


def test_matches_cuda_core_fp32_trajectory():
    """A whole trajectory (refresh, 10 fused steps, Metropolis) on the tensor
    cores agrees with the FP32 row kernels and the FP64 engine in dH."""
    nc, dims = 32, [2, 2, 2]
    O, u, pi, beta = setup(nc, dims, 99)
    res = {}
    for path, prec in [(2, "fp32"), (1, "fp32"), (0, "fp64")]:
        with ab.Engine(nc, dims, beta=beta, dt=0.005, level=8, precision=prec, kernel_path=path, seed=7) as e:
            e.set_links(u)
            r = e.trajectory(10)
            res[path] = r
    assert abs(res[2]["dh"] - res[0]["dh"]) < 1e-3
    assert abs(res[1]["dh"] - res[0]["dh"]) < 1e-3
    assert res[2]["h_old"] == pytest.approx(res[0]["h_old"], rel=1e-6)


@pytest.mark.parametrize("nc,dims,precision", [(16, [2, 3, 2], "fp64"), (32, [2, 2, 3], "fp64"),
                                               (64, [2, 3], "fp64"), (32, [2, 2, 3], "fp32")])
def test_large_nc_reductions_vs_oracle(nc, dims, precision):
    """CTA-per-site plaquette sums and CTA-per-link kinetic / UViol sums
    (NC >= 16), accumulated in FP64 for either storage precision."""
    O, u, pi, beta = setup(nc, dims, 5 * nc)
    Pi = fields.momenta(nc, O.vol * O.dim, beta, np.random.default_rng(nc + 1), O)
    if precision == "fp32":  # compare on the FP32-rounded inputs the engine actually holds
        u = u.astype(np.complex64).astype(np.complex128)
        pi = pi.astype(np.complex64).astype(np.complex128)
        Pi = Pi.astype(np.complex64).astype(np.complex128)
    with ab.Engine(nc, dims, beta=beta, precision=precision) as e:
        e.set_links(u)
        e.set_momenta(pi, 0)
        e.set_momenta(Pi, 1)
        assert e.EnergyMag() == pytest.approx(O.EnergyMag(u), rel=1e-12)
        t, s = e.PlaqExp()
        assert t + s == pytest.approx(O.EnergyMag(u), rel=1e-12)
        assert e.simpleenergyEl(0) == pytest.approx(O.simpleenergyEl(pi), rel=1e-12)
        assert e.EnergyEl() == pytest.approx(O.EnergyEl(pi, Pi), rel=1e-12)
        assert e.UViol() == pytest.approx(O.UViol(u), rel=1e-6, abs=1e-18 * O.vol * O.dim)


def test_path_validation():
    with pytest.raises(ab.AskjaError):
        ab.Engine(32, [2, 2], beta=1.0, precision="fp64", kernel_path=2)
    with pytest.raises(ab.AskjaError):
        ab.Engine(24, [2, 2], beta=1.0, precision="fp32", kernel_path=2)
    with pytest.raises(ab.AskjaError):
        ab.Engine(8, [2, 2], beta=1.0, precision="fp32", kernel_path=2)
    with pytest.raises(ab.AskjaError):
        ab.Engine(32, [4], beta=1.0, precision="fp32", kernel_path=2)
    with ab.Engine(32, [2, 2], beta=1.0, precision="fp32") as e:
        ab.set_tuning(e, {"path": 2})
        ab.set_tuning(e, {"path": 1})
    with ab.Engine(32, [2, 2], beta=1.0, precision="fp64") as e:
        with pytest.raises(ab.AskjaError):
            ab.set_tuning(e, {"path": 2})


def test_trajectories_stay_unitary_with_gated_gram_schmidt():
    """Tensor-core trajectories (graph replays): the link update keeps U' as
    unitary as U and the engine re-orthonormalises U before every 10th
    trajectory, so the defect stays at FP32 rounding over many trajectories."""
    nc, dims = 32, [2, 2, 2]
    O, u, pi, beta = setup(nc, dims, 5)
    with ab.Engine(nc, dims, beta=beta, dt=0.005, level=8, precision="fp32", kernel_path=2, seed=3) as e:
        e.set_links(u)
        last, log = e.run_trajectories(12, 10, use_graph=True)
        assert last["n_tot"] == 12
        assert np.all(np.isfinite(log))
        assert unitarity(e.get_links()) < 3e-6
        assert unitarity(e.get_saved_links()) < 3e-6
        # dH stays small at this step size
        assert np.abs(log[:, 2]).max() < 1.0


def test_bounded_wait_gives_up_and_context_survives():
    """The tensor-core path's bounded wait on an mbarrier that nothing
    completes (askja_tc_wait_selftest, one CTA, no tensor-core instruction
    issued): the wait ends after its limit, the next synchronising call
    reports it, and the context then runs normal trajectories."""
    nc, dims = 32, [2, 2, 2]
    with ab.Engine(nc, dims, beta=2.0 * nc * nc, dt=0.005, level=8, precision="fp32", kernel_path=2, seed=3) as e:
        e.hot_start(5)
        e.tc_wait_selftest(100_000)
        with pytest.raises(ab.AskjaError) as ex:
            e.sync()
        assert ex.value.code == -2 and "gave up waiting" in str(ex.value)
        e.sync()  # the error is reported once
        r = e.trajectory(3)
        assert np.isfinite(r["dh"])
    with ab.Engine(nc, dims, beta=2.0 * nc * nc, precision="fp32", kernel_path=1) as e:
        with pytest.raises(ab.AskjaError):
            e.tc_wait_selftest(1000)  # only on the tensor-core mapping


def test_su16_tensor_cores_match_row_kernel_trajectory():
    """SU(16) on the padded tensor-core shape against the FP32 row kernels and
    the FP64 engine: one whole trajectory, same dH to 1e-3."""
    nc, dims = 16, [2, 2, 3]
    O, u, pi, beta = setup(nc, dims, 161)
    res = {}
    for path, prec in [(2, "fp32"), (1, "fp32"), (0, "fp64")]:
        with ab.Engine(nc, dims, beta=beta, dt=0.005, level=8, precision=prec, kernel_path=path, seed=7) as e:
            e.set_links(u)
            res[path] = e.trajectory(10)
    assert abs(res[2]["dh"] - res[0]["dh"]) < 1e-3
    assert abs(res[1]["dh"] - res[0]["dh"]) < 1e-3
