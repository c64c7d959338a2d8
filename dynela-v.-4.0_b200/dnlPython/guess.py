"""Learned Newton initial guess of the radial return: harvest training pairs
from the engine's own returns, train the network on the GPU, and measure
what it changes.

    pairs, stats = harvest(descs, capacity=10_000_000, stride=2000, max_incs=3000)
    net, losses = train(pairs, epochs=8)
    with Engine(desc) as e:
        e.init(); e.set_guess_network(net); e.set_mode(_abi.MODE_GUESS); e.run()

Device buffers are torch tensors (plumbing); every kernel is the engine's
(include/dnlgpu.h: dnl_engine_set_harvest, dnl_mlp_train, dnl_mlp_forward).
"""
import ctypes

import numpy as np

from . import _abi
from .engine import Engine


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _abi.EngineUnavailable("the learned guess needs a CUDA device")
    return torch


def harvest(descs, capacity, stride, max_incs=0, t_pause=np.inf, scope=_abi.GUESS_ALL, info=None):
    """Run `descs` (one model or a batch) with the plain return and keep one
    yielding point of `scope` in `stride` as a (5 inputs, r = gamma /
    gamma_max, gamma, gamma_max) pair.  Returns a device tensor [n, 8] and the Newton statistics
    of the run (Engine.newton_stats).  The points are chosen by a hash of
    (point, increment), so the set is reproducible as long as it fits in
    `capacity`; past it, which points are kept depends on the order of the
    appends.  info (a dict), if given, receives "candidates": the points that
    passed the stride, kept or not."""
    torch = _torch()
    buf = torch.zeros((int(capacity), _abi.MLP_PAIR_WORDS), dtype=torch.float32, device="cuda")
    with Engine(descs) as e:
        e.init()
        e.set_harvest(buf.data_ptr(), buf.shape[0], stride)
        e.set_guess_scope(scope)
        e.set_mode(_abi.MODE_HARVEST)
        e.run(t_pause=t_pause, max_incs=max_incs, check=False)
        n = e.harvest_count()
        stats = e.newton_stats()
    if info is not None:
        info["candidates"] = int(n)
    n = min(int(n), int(capacity))
    # the kernels append pairs in whatever order their atomics resolve: sort
    # the rows (lexicographically, by stable passes from the last word) so
    # that training on them is reproducible
    pairs = buf[:n].clone()
    for c in range(_abi.MLP_PAIR_WORDS - 1, -1, -1):
        pairs = pairs[torch.sort(pairs[:, c], stable=True).indices]
    return pairs, stats


def initial_network(x, r, seed=1):
    """He-initialised network whose input normalisation maps the 0.1-99.9 %
    range of the harvested inputs x [n, 5] to [-1, 1] and holds inputs outside
    it at the edge (in_clip = 1: a model whose inputs leave the training
    range, a finer mesh's time step for instance, is not extrapolated), and
    whose output bias is the mean target."""
    rng = np.random.default_rng(seed)
    H, K, NIN = _abi.MLP_HIDDEN, 16, _abi.MLP_IN
    lo, hi = np.percentile(x, [0.1, 99.9], axis=0)
    w1 = np.zeros((H, K), np.float32)
    w1[:, :NIN] = rng.normal(0, np.sqrt(2.0 / NIN), (H, NIN))
    d = dict(w1=w1, b1=np.zeros(H, np.float32), w2=rng.normal(0, np.sqrt(2.0 / H), (H, H)).astype(np.float32),
             b2=np.zeros(H, np.float32), w3=rng.normal(0, np.sqrt(2.0 / H), (H, H)).astype(np.float32),
             b3=np.zeros(H, np.float32), w4=(0.1 * rng.normal(0, np.sqrt(1.0 / H), H)).astype(np.float32),
             b4=np.float32(np.mean(r)), in_mean=((lo + hi) / 2).astype(np.float32),
             in_scale=(2.0 / np.maximum(hi - lo, 1e-6)).astype(np.float32), in_clip=np.float32(1.0))
    return _abi.Mlp.from_dict(d)


def first_yield(pairs):
    """The pairs of points yielding for the first time (eps_p = 0): the
    points the reference starts from gamma = 1e-8."""
    return pairs[pairs[:, 1] == 0.0]


def train(pairs, epochs=8, batch_tiles=128, learning_rate=1e-3, seed=20261203, net=None, log_target=False):
    """Adam training of the network on harvested pairs (device tensor [n, 8])
    by the engine's kernels, on r = gamma / gamma_max (log_target: on ln r,
    for points whose r spans decades, such as first-yield points).  Returns
    the trained dnl_mlp and the per-epoch mean squared error."""
    torch = _torch()
    lib = _abi.load_library()
    x = pairs[:, :_abi.MLP_IN].contiguous()
    # r past 2 (a yield stress that fell a long way during the increment) is
    # rare and heavy-tailed; the guess is clamped to [0, 2] gamma_max anyway
    r = pairs[:, 5].clamp(1e-6 if log_target else 0.0, 2.0)
    r = (torch.log(r) if log_target else r).contiguous()
    n = x.shape[0]
    if net is None:
        g = torch.Generator(device=pairs.device).manual_seed(int(seed) % (2 ** 63))
        pick = torch.randperm(n, device=pairs.device, generator=g)[:200000]
        net = initial_network(x[pick].cpu().numpy(), r[pick].cpu().numpy())
    net.out_exp = 1.0 if log_target else 0.0
    hist = (ctypes.c_float * max(1, epochs))()
    rc = lib.dnl_mlp_train(ctypes.byref(net), x.data_ptr(), r.data_ptr(), n, int(epochs), int(batch_tiles),
                           float(learning_rate), int(seed), hist, None)
    if rc != 0:
        raise _abi.EngineError(rc, lib.dnl_engine_last_error(None).decode())
    return net, list(hist[:epochs])


def predict(net, x):
    """Network outputs for inputs x (device tensor [n, 5])."""
    torch = _torch()
    lib = _abi.load_library()
    x = x.contiguous().float()
    y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
    rc = lib.dnl_mlp_forward(ctypes.byref(net), x.data_ptr(), x.shape[0], y.data_ptr(), None)
    if rc != 0:
        raise _abi.EngineError(rc, lib.dnl_engine_last_error(None).decode())
    return y


def compare(desc, net, warm_incs, incs, scope=_abi.GUESS_ALL):
    """Run `desc` to increment warm_incs with the plain return, then `incs`
    more increments once with the warm start (counted) and once from the
    network's guess (for the points of `scope`), from the same state.
    Returns, per mode, the Newton evaluations per yielding point and per point
    of the scope, the FP64 re-solves and the element-pass time per increment,
    and the relative differences of the guessed run's stress, plastic strain
    and coordinates from the plain run's.  `perfect_guess_bound`: what a
    perfect network that costs nothing could save at most — every point of
    the scope down to the one evaluation that confirms the root — as a
    fraction of all the return's evaluations in the plain run."""
    out, ref = {}, None
    for name, mode in (("plain", _abi.MODE_STATS), ("guess", _abi.MODE_GUESS)):
        with Engine(desc) as e:
            e.init()
            if warm_incs:
                e.run(max_incs=warm_incs)
            e.set_guess_network(net)
            e.set_guess_scope(scope)
            e.set_mode(mode)
            e.newton_stats(reset=True)
            e.set_timing(True)
            e.run(max_incs=incs)
            tm = e.timings()
            ev, pl, sc, sev = e.newton_stats()
            c = e.control()
            out[name] = dict(evals_per_point=ev / max(pl, 1), yielding_points=pl, scope_points=sc,
                             evals_per_scope_point=sev / max(sc, 1),
                             fp64_resolve_rate=c["fp64_resolves"] / max(pl, 1),
                             element_ms=tm["element_ms"] / max(incs, 1))
            if name == "plain":
                out["perfect_guess_bound"] = dict(evaluations_saved=int(sev - sc),
                                                  fraction_of_all_evaluations=(sev - sc) / max(ev, 1))
            ips = e.ips()
            s = ips[_abi.IP_STRESS:_abi.IP_STRESS + 6]
            ep = ips[_abi.IP_EPSP]
            x = e.nodes(_abi.NODE_COORDS)
            if ref is None:
                ref = (s, ep, x)
            else:
                out["guess_vs_plain"] = dict(
                    stress=float(np.abs(s - ref[0]).max() / np.abs(ref[0]).max()),
                    max_epsp=float(abs(ep.max() - ref[1].max()) / max(ref[1].max(), 1e-30)),
                    epsp=float(np.abs(ep - ref[1]).max() / max(np.abs(ref[1]).max(), 1e-30)),
                    coords=float(np.abs(x - ref[2]).max() / np.abs(ref[2]).max()))
    return out
