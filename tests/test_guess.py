"""The learned Newton initial guess of the radial return: the network's
kernels (BF16 tensor-core products, FP32 accumulation) against the numpy
oracle of oracle/mlp_ref.py, its training, and the element pass that starts
the return from the network's guess (it converges to the same returned state)."""
import ctypes

import numpy as np
import pytest

import helpers
from helpers import _abi, meshes
import mlp_ref


def net_struct(d):
    return _abi.Mlp.from_dict(d)


def test_oracle_backward_matches_finite_differences():
    """The oracle's analytic gradient (without the BF16 roundings, in FP64)
    against central differences of its own loss."""
    rng = np.random.default_rng(3)
    net = {k: np.asarray(v, np.float64) for k, v in mlp_ref.random_net(5).items()}
    x = rng.normal(0, 1, (40, 5))
    t = rng.normal(0, 1, 40)
    g, _ = mlp_ref.gradients(net, x, t, rounding=False)

    def loss():
        y, _ = mlp_ref.forward(net, x, rounding=False)
        return np.mean((y - t) ** 2)

    for name, idx in (("w1", (3, 2)), ("b1", (7,)), ("w2", (10, 33)), ("b2", (5,)), ("w3", (60, 1)), ("b3", (0,)),
                      ("w4", (12,)), ("b4", ())):
        a = net[name]
        h = 1e-6
        if a.ndim == 0:
            net[name] = a + h
            lp = loss()
            net[name] = a - h
            lm = loss()
            net[name] = a
        else:
            a[idx] += h
            lp = loss()
            a[idx] -= 2 * h
            lm = loss()
            a[idx] += h
        fd = (lp - lm) / (2 * h)
        an = float(np.asarray(g[name])[idx]) if np.ndim(g[name]) else float(g[name])
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (name, fd, an)


def test_bf16_rounding_of_the_oracle():
    a = np.array([1.0, 1.00390625, 1.0078125, -3.1415927, 1e-30, 65504.0], np.float32)
    b = mlp_ref.bf16(a)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties go to the even mantissa (1.0)
    assert b[0] == 1.0 and b[1] == 1.0 and b[2] == np.float32(1.0078125)
    assert abs(b[3] + 3.140625) < 1e-7


def test_network_struct_round_trip():
    net = mlp_ref.random_net(9)
    back = net_struct(net).to_dict()
    for k, v in net.items():
        assert np.array_equal(np.asarray(back[k]), np.asarray(v, np.float32)), k


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("n,clip", [(1, 0.0), (128, 0.0), (1000, 0.0), (1000, 1.0)])
def test_forward_matches_oracle(n, clip):
    """Network outputs on the tensor cores against the oracle; with in_clip the
    normalised inputs (about a third of them past +-1 here) are held at +-clip."""
    import torch
    lib = _abi.load_library()
    net = mlp_ref.random_net(11)
    net["in_mean"] = np.array([1.0, 0.1, 2.0, 0.3, -10.0], np.float32)
    net["in_scale"] = np.array([0.5, 3.0, 0.4, 2.0, 0.2], np.float32)
    net["in_clip"] = np.float32(clip)
    rng = np.random.default_rng(n)
    x = (net["in_mean"] + rng.normal(0, 1, (n, 5)) / net["in_scale"]).astype(np.float32)
    dx, dy = _dev(x), torch.zeros(n, dtype=torch.float32, device="cuda")
    s = net_struct(net)
    assert lib.dnl_mlp_forward(ctypes.byref(s), dx.data_ptr(), n, dy.data_ptr(), None) == 0, \
        lib.dnl_engine_last_error(None).decode()
    y = dy.cpu().numpy()
    y_ref, _ = mlp_ref.forward(net, x)
    assert np.abs(y - y_ref).max() <= 5e-3 * (1.0 + np.abs(y_ref).max())
    if clip > 0.0:
        # the same as feeding the inputs already held at the edge, unheld
        xc = net["in_mean"] + np.clip((x - net["in_mean"]) * net["in_scale"], -clip, clip) / net["in_scale"]
        y_c, _ = mlp_ref.forward(dict(net, in_clip=np.float32(0.0)), xc.astype(np.float32))
        assert np.abs(y_ref - y_c).max() <= 1e-3 * (1.0 + np.abs(y_c).max())


@pytest.mark.gpu
def test_gradients_match_oracle():
    import torch
    lib = _abi.load_library()
    net = mlp_ref.random_net(21)
    rng = np.random.default_rng(22)
    n = 700
    x = rng.normal(0, 1, (n, 5)).astype(np.float32)
    t = np.tanh(x[:, 0] - 0.5 * x[:, 1] * x[:, 2]).astype(np.float32)
    s, g = net_struct(net), _abi.Mlp()
    loss = ctypes.c_float()
    assert lib.dnl_mlp_gradients(ctypes.byref(s), _dev(x).data_ptr(), _dev(t).data_ptr(), n, ctypes.byref(g),
                                 ctypes.byref(loss), None) == 0, lib.dnl_engine_last_error(None).decode()
    torch.cuda.synchronize()
    gg = g.to_dict()
    g_ref, l_ref = mlp_ref.gradients(net, x, t)
    assert abs(loss.value - l_ref) <= 2e-3 * l_ref
    for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4"):
        a, b = np.asarray(gg[k], np.float64), np.asarray(g_ref[k], np.float64)
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-7, k


@pytest.mark.gpu
def test_training_fits_a_smooth_function():
    lib = _abi.load_library()
    rng = np.random.default_rng(31)
    n = 40000
    x = rng.uniform(-1, 1, (n, 5)).astype(np.float32)
    t = (0.5 + 0.3 * np.sin(2 * x[:, 0]) * x[:, 1] - 0.2 * x[:, 2] ** 2).astype(np.float32)
    net = mlp_ref.random_net(32)
    s = net_struct(net)
    hist = (ctypes.c_float * 20)()
    assert lib.dnl_mlp_train(ctypes.byref(s), _dev(x).data_ptr(), _dev(t).data_ptr(), n, 20, 32, 2e-3, 7, hist,
                             None) == 0, lib.dnl_engine_last_error(None).decode()
    h = np.array(hist[:])
    assert h[-1] < 0.05 * h[0] and h[-1] < 2e-3
    # the trained weights in the oracle reproduce the loss the device reports
    y_ref, _ = mlp_ref.forward(s.to_dict(), x)
    assert np.mean((y_ref - t) ** 2) < 1.5 * h[-1]


def _engine(desc):
    from dnlPython.engine import Engine
    return Engine(desc)


def _bar():
    return meshes.taylor_3d(n_core=4, n_ring=3, n_axial=40, precision=_abi.PREC_MIXED)


@pytest.mark.gpu
def test_harvested_pairs_are_consistent():
    import torch
    buf = torch.zeros((200000, _abi.MLP_PAIR_WORDS), dtype=torch.float32, device="cuda")
    with _engine(_bar()) as e:
        e.init()
        e.set_harvest(buf.data_ptr(), buf.shape[0], 1)
        e.set_mode(_abi.MODE_HARVEST)
        e.run(max_incs=40)
        n = min(e.harvest_count(), buf.shape[0])  # the count goes on past the buffer's capacity
        evals, plastic, in_scope, _ = e.newton_stats()
    assert n > 1000 and plastic >= n and in_scope == plastic and evals >= plastic
    p = buf[:n].cpu().numpy()
    x, r, gamma, gmax = p[:, :5], p[:, 5], p[:, 6], p[:, 7]
    # r = gamma / gamma_max, gamma_max the bound of a yield stress that does not
    # fall during the increment: thermal softening or a lower strain rate than
    # the previous increment's can take gamma past it
    assert np.all(gmax > 0) and np.all(r >= 0) and np.all(np.isfinite(r)) and np.mean(r > 1.0) < 0.2
    assert np.allclose(gamma, r * gmax, rtol=1e-5, atol=0)
    assert np.all(x[:, 0] > 0) and np.all((x[:, 3] > 0) & (x[:, 3] < 1)) and np.all(np.isfinite(x))


@pytest.mark.gpu
@pytest.mark.parametrize("scope", [_abi.GUESS_ALL, _abi.GUESS_FIRST_YIELD], ids=["all", "first-yield"])
def test_guess_mode_reaches_the_plain_return(scope):
    """From the same state, one increment with the network's first iterate
    (an untrained network: a poor guess) and one with the warm start return
    the same state to the FP32 Newton tolerance."""
    out = {}
    for mode in (_abi.MODE_STATS, _abi.MODE_GUESS, _abi.MODE_PLAIN):
        with _engine(_bar()) as e:
            e.init()
            e.run(max_incs=60)
            e.set_guess_network(net_struct(mlp_ref.random_net(41)))
            e.set_guess_scope(scope)
            e.set_mode(mode)
            e.newton_stats(reset=True)
            e.run(max_incs=1)
            out[mode] = (e.ips(), e.nodes(_abi.NODE_COORDS), e.newton_stats())
    ip_s, x_s, st_s = out[_abi.MODE_STATS]
    ip_g, x_g, st_g = out[_abi.MODE_GUESS]
    ip_p, x_p, _ = out[_abi.MODE_PLAIN]
    assert st_s[1] > 0 and st_g[1] == st_s[1] and st_g[2] == st_s[2] > 0
    assert (st_g[2] == st_g[1]) if scope == _abi.GUESS_ALL else (st_g[2] < st_g[1])
    # gamma converges to the return's absolute step tolerance (1e-8, Element.C:419,547):
    # it is compared per point on that scale; the plastic strain rate
    # gamma sqrt(2/3) / dt and the yield stress through its rate term
    # C ln(rate) amplify that tolerance at points that have just yielded (tiny
    # gamma), so they get a looser bound; every other component is held to 1e-4
    # of its largest value
    # The stress is held to what the return's own tolerance allows: the return
    # sets s = dev* (1 - 2G gamma / |dev*|) + p (Element.C:587-600), so a
    # point's stress moves by at most 2G |d gamma| (then an orthogonal
    # rotation); on top of that FP32 rounding, 2e-6 of the largest stress.
    loose = (_abi.IP_DEPSP, _abi.IP_GAMMA, _abi.IP_YIELD)
    stress = list(range(_abi.IP_STRESS, _abi.IP_STRESS + 6))
    other = [c for c in range(_abi.IP_NCOMP) if c not in loose and c not in stress]
    twoG = meshes.COPPER["young"] / (1.0 + meshes.COPPER["poisson"])
    for a, b in ((ip_g, ip_s), (ip_s, ip_p)):
        dgamma = np.abs(a[_abi.IP_GAMMA] - b[_abi.IP_GAMMA])
        assert np.all(dgamma <= 4e-8 + 1e-5 * np.abs(b[_abi.IP_GAMMA]))
        ds = np.abs(a[stress] - b[stress]).max(axis=0)
        assert np.all(ds <= 1.5 * twoG * dgamma + 2e-6 * np.abs(b[stress]).max()), \
            (ds / (1.5 * twoG * dgamma + 2e-6 * np.abs(b[stress]).max())).max()
        assert helpers.field_errors(a[other], b[other]).max() < 1e-4
        y_a, y_b = a[_abi.IP_YIELD], b[_abi.IP_YIELD]
        assert np.abs(y_a - y_b).max() <= 5e-3 * np.abs(y_b).max()
    assert helpers.rel_err(x_g, x_s) < 1e-9


@pytest.mark.gpu
def test_trained_guess_cuts_first_yield_iterations():
    """Trained on first-yield returns of a few bars (ln r targets), the network
    starts the return of points yielding for the first time closer to the
    root than the reference's gamma = 1e-8: fewer yield-function evaluations
    at those points, the same returned state to the return's tolerance."""
    from dnlPython import guess
    pairs, st = guess.harvest(meshes.taylor_batch(n=8, seed=5, elems=(2000, 8000)), capacity=2_000_000, stride=1,
                              max_incs=1500, scope=_abi.GUESS_FIRST_YIELD)
    assert pairs.shape[0] > 100000
    net, hist = guess.train(pairs, epochs=20, batch_tiles=64, log_target=True)
    assert hist[-1] < 0.5 * hist[0]
    res = guess.compare(meshes.taylor_3d(n_core=6, n_ring=8, n_axial=80, speed=250000.0), net, 0, 300,
                        scope=_abi.GUESS_FIRST_YIELD)
    plain, guessed = res["plain"], res["guess"]
    assert plain["scope_points"] > 10000 and guessed["scope_points"] == plain["scope_points"]
    assert guessed["evals_per_scope_point"] < 0.85 * plain["evals_per_scope_point"]
    assert res["guess_vs_plain"]["stress"] < 2e-3 and res["guess_vs_plain"]["max_epsp"] < 1e-4
