"""A pass split across ranks by shell pixels (hammurabix_b200.sharded and
hxg_shell_integrate_device / hxg_shell_merge_device).

CPU (gloo, 2 ranks): the exchange logic with a stand-in integrator that
keeps the library's contract (shell maps zero outside the shard, a shell's
values depend on the accumulated FD map of the inner shells, a linear
merge): both ranks end with the single-process outputs.

GPU (one device): the shards of a pass emulated one after another in one
process -- each shard's shell maps summed the way the all-reduce sums them --
against the unsplit hxg_write_grid_device: to rounding in FP64 (a shard has
fewer pixels, so it may split each ray over more lanes, which regroups the
sums) and to the FP32C tolerance.

The sharded adjoint (sharded.adjoint_sharded, hxg_adjoint_shard_*): on CPU
the two gloo ranks run its exchange with the stand-in's adjoint; on the GPU
emulated shards, one handle each, against hxg_adjoint_device.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from conftest import rel_err  # noqa: E402
from hammurabix_b200 import abi, sharded, workloads as W  # noqa: E402


def _block_log2(npix, n):
    """The library's shard block size (shard_block_log2, hxg_api.cu)."""
    L = 11
    while L > 5 and (npix >> L) < 8 * n:
        L -= 1
    return L


def _owned(npix, r, n):
    """NESTED pixels of shard r of n: the blocks b of 2^L pixels with
    b % n == r (the library's shard_nest, written out)."""
    nest = np.arange(npix)
    return (nest >> _block_log2(npix, n)) % n == r


class FakeIntegrator:
    """Per-shell stand-in with the library's sharding contract."""

    def shell_integrate_device(self, obs, s, shard, nshards, fd, tmp):
        n = abi.npix(obs.nside_shell[s])
        own = torch.from_numpy(_owned(n, shard, nshards))
        inner = float(fd.sum()) if fd is not None else 0.0   # needs the complete FD map
        base = 1.0 + s + 0.01 * torch.arange(n, dtype=torch.float64)
        for k, t in enumerate(tmp):
            if t is None:
                continue
            t.zero_()
            t[own] = (k + 1) * base[own] + 1e-3 * inner

    def shell_integrate_multi_device(self, passes, s, shard, nshards, fd, dm_t, fd_t, iqu):
        n = abi.npix(passes[0].nside_shell[s])
        own = torch.from_numpy(_owned(n, shard, nshards))
        inner = float(fd.sum()) if fd is not None else 0.0
        base = 1.0 + s + 0.01 * torch.arange(n, dtype=torch.float64)
        for k, t in enumerate([dm_t, fd_t]):
            t.zero_()
            t[own] = (k + 1) * base[own]
        for f, o in enumerate(passes):
            for j, t in enumerate(iqu[f]):
                t.zero_()
                t[own] = (3 + j) * base[own] * (1 + 0.1 * f) + 1e-3 * inner * o.do_fd

    def shell_merge_device(self, obs, s, tmp, outs):
        for t, o in zip(tmp, outs):
            if t is None or o is None:
                continue
            g = torch.Generator().manual_seed(len(o) * 7919 + len(t))
            o += torch.rand(len(o), len(t), generator=g, dtype=torch.float64) @ t

    # the sharded adjoint's contract: a shell's terms come from this shard's
    # pixels only and depend on the complete dL/d(FD map) of the outer
    # shells; the gradient accumulators are sums over the pixels
    def adjoint_shard_begin(self, obs, shard, nshards):
        self._shard = (shard, nshards)
        self._acc = torch.zeros(8 + 4 * 5, dtype=torch.float64)

    def adjoint_shard_shell(self, obs, s, g_dm, g_fdmap, g_is, g_qs, g_us, inc):
        n = abi.npix(obs.nside_shell[s])
        own = torch.from_numpy(_owned(n, *self._shard)).double()
        w = own * (1.0 + s + 0.01 * torch.arange(n, dtype=torch.float64))
        level = 1.0 + 1e-3 * float(g_fdmap.sum()) + 1e-4 * float(g_is.sum())
        g = torch.Generator().manual_seed(len(inc) * 104729 + n)
        inc.zero_()
        inc += (torch.rand(len(inc), n, generator=g, dtype=torch.float64) @ w) * level
        g2 = torch.Generator().manual_seed(n)
        self._acc += (torch.rand(len(self._acc), n, generator=g2, dtype=torch.float64) @ w) * level

    def adjoint_shard_finish(self, params, b, ne):
        params.copy_(self._acc[:8])
        for k, t in enumerate(b):
            t.copy_(self._acc[8 + 5 * k:13 + 5 * k])
        ne.copy_(self._acc[23:28])


def _obs():
    return W.make_obs([4, 8, 8], 20.0, 0.1, freq_ghz=1.4)


def _run(world, rank, reduce_sum, reduce_root=None):
    o = _obs()
    out_n = abi.npix(8)
    outs = {k: torch.zeros(out_n, dtype=torch.float64) for k in sharded.MAPS}
    tmp = {k: torch.zeros(out_n, dtype=torch.float64) for k in sharded.MAPS}
    sharded.write_grid_sharded(FakeIntegrator(), o, outs, tmp, rank, world, reduce_sum,
                               reduce_root)
    return {k: v.numpy().copy() for k, v in outs.items()}


def _passes():
    return W.frequency_passes(W.make_obs([4, 8, 8], 20.0, 0.1, freq_ghz=1.4), [0.408, 1.4, 30.0])


def _run_passes(world, rank, reduce_sum, reduce_root=None):
    ps = _passes()
    out_n = abi.npix(8)
    z = lambda n: torch.zeros(n, dtype=torch.float64)
    outs = [{k: z(out_n) for k in sharded.MAPS} for _ in ps]
    sharded.write_passes_sharded(FakeIntegrator(), ps, outs, sharded.make_shell_maps(out_n, z),
                                 rank, world, reduce_sum, reduce_root)
    return [{k: v.numpy().copy() for k, v in o.items()} for o in outs]


def _run_adjoint(world, rank, reduce_sum):
    o = _obs()
    z = lambda n: torch.zeros(n, dtype=torch.float64)
    ndm, nfd, nsy = abi.obs_output_sizes(o)
    gen = torch.Generator().manual_seed(3)
    g = {k: torch.rand(c, generator=gen, dtype=torch.float64)
         for k, c in zip(sharded.MAPS, (ndm, nfd, nsy, nsy, nsy))}
    grads = {"params": z(8), "b": [z(5) for _ in range(3)], "ne": z(5)}
    sharded.adjoint_sharded(FakeIntegrator(), o, g, grads, rank, world, reduce_sum, z)
    return np.concatenate([grads["params"].numpy()] + [t.numpy() for t in grads["b"]] +
                          [grads["ne"].numpy()])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import torch.distributed as dist
    from hammurabix_b200 import replicas
    w, r, _ = replicas.init("gloo", 60)
    red = lambda t: dist.all_reduce(t)
    root = lambda t: dist.reduce(t, dst=0)
    q.put((r, (_run(w, r, red, root), _run_passes(w, r, red, root), _run_adjoint(w, r, red))))
    replicas.finish(w)


def test_two_gloo_ranks_reproduce_the_single_process_pass():
    """One pass (per-shell exchange), three fused passes of the Pipeline's
    order and the sharded adjoint of the one pass (per-shell exchange of
    the FD-map gradient, all-reduced gradients), on two ranks, against one
    process: every rank ends with the single process's gradients; rank 0 ends with
    every map of the single process (the DM and Stokes maps reduced onto
    it), every rank with the complete FD map, and rank 1's DM and Stokes
    maps stay its own shard's partial maps (no all-reduce at the end)."""
    single = _run(1, 0, None)
    single_multi = _run_passes(1, 0, None)
    single_adj = _run_adjoint(1, 0, None)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        one, multi, adj = got[r]
        # the sharded adjoint: every rank ends with the full gradient
        assert np.abs(single_adj).max() > 0
        assert rel_err(adj, single_adj) <= 1e-12, r
        for k in sharded.MAPS:
            assert np.abs(single[k]).max() > 0, k
            if r == 0 or k == "fd":
                assert rel_err(one[k], single[k]) <= 1e-12, (r, k)
            else:
                assert rel_err(one[k], single[k]) > 1e-3, (r, k)
        for p, (a, b) in enumerate(zip(multi, single_multi)):
            for k in sharded.MAPS:
                if sharded.requested(_passes()[p])[k]:
                    assert np.abs(b[k]).max() > 0, (p, k)
                    if r == 0 or k == "fd":
                        assert rel_err(a[k], b[k]) <= 1e-12, (r, p, k)
    # rank 1 keeps its own shard's part of DM / I / Q / U, a nonzero share
    for k in ("dm", "is", "qs", "us"):
        assert np.abs(got[1][0][k]).max() > 0, k


def test_shards_partition_every_shell():
    """shard_nest (hxg_integrate.cuh) maps each shard's local pixels onto its
    blocks; over all shards every NESTED pixel is taken exactly once."""
    for npix in (12, 48, 192, 768, 12 * 64 ** 2, 12 * 256 ** 2):
        for n in (1, 2, 3, 8):
            seen = np.zeros(npix, dtype=int)
            L = _block_log2(npix, n)
            nblk = (npix + (1 << L) - 1) >> L
            for r in range(n):
                local = np.arange((nblk + n - 1 - r) // n << L if n > 1 else npix)
                nest = local if n == 1 else (((local >> L) * n + r) << L) + (local & ((1 << L) - 1))
                nest = nest[nest < npix]
                assert np.all(_owned(npix, r, n)[nest])
                seen[nest] += 1
            assert np.all(seen == 1)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32c", 1e-5)])
@pytest.mark.parametrize("nshards", [2, 3])
def test_emulated_shards_match_the_unsplit_pass(fields32, precision, tol, nshards):
    from hammurabix_b200.integrator import Integrator
    dev = torch.device("cuda", 0)
    # one stream for the library and torch's own work on the maps (a null
    # stream handle would leave the library on its own stream)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    passes = [W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=0.408),
              W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=23.0, do_fd=False)]
    with Integrator(precision) as integ:
        integ.set_stream(stream.cuda_stream)
        integ.set_models(W.grid_models())
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        for o in passes:
            ndm, nfd, nsy = abi.obs_output_sizes(o)
            z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev) if n else None
            ref = [z(ndm), z(nfd), z(nsy), z(nsy), z(nsy)]
            integ.write_grid_device(o, *ref)
            req = sharded.requested(o)
            need = sharded.shell_maps_needed(o)
            nmax = abi.npix(max(o.nside_shell[s] for s in range(o.total_shell)))
            # per-shard outputs; the FD output is shared (every rank holds the same)
            outs = [[z(ndm), None, z(nsy), z(nsy), z(nsy)] for _ in range(nshards)]
            fd = z(nfd)
            for s in range(o.total_shell):
                n = abi.npix(o.nside_shell[s])
                shard_tmp = []
                for r in range(nshards):
                    t = [z(nmax)[:n] if need[k] else None for k in sharded.MAPS]
                    integ.shell_integrate_device(o, s, r, nshards, fd, t)
                    shard_tmp.append(t)
                fd_sum = None
                if req["fd"]:
                    fd_sum = sum(t[1] for t in shard_tmp)       # the per-shell all-reduce
                for r in range(nshards):
                    t = list(shard_tmp[r])
                    out_r = list(outs[r])
                    if req["fd"]:
                        # every rank merges the summed FD map; one FD output
                        # stands for all of them (they are identical)
                        t[1] = fd_sum
                        out_r[1] = fd if r == 0 else z(nfd)
                    integ.shell_merge_device(o, s, t, out_r)
            integ.sync()
            got = [None] * 5
            got[1] = fd
            for j in (0, 2, 3, 4):
                if outs[0][j] is not None:
                    got[j] = sum(outs[r][j] for r in range(nshards))  # the final all-reduce
            for j, k in enumerate(sharded.MAPS):
                if not req[k]:
                    continue
                a, b = got[j].cpu().numpy(), ref[j].cpu().numpy()
                assert rel_err(a, b) <= tol, (k, rel_err(a, b))
                assert np.abs(b).max() > 0, k


@pytest.mark.gpu
@pytest.mark.parametrize("nshards", [1, 3])
def test_emulated_shards_of_fused_passes(fields32, nshards):
    """Three fused passes (hxg_shell_integrate_multi_device) split into
    shards run one after another, against the passes one by one."""
    from hammurabix_b200.integrator import Integrator
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    passes = W.frequency_passes(W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=0.408),
                                [0.408, 1.4, 30.0])
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev) if n else None
    with Integrator("fp32c") as integ:
        integ.set_stream(stream.cuda_stream)
        integ.set_models(W.grid_models())
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        ref = []
        for o in passes:
            ndm, nfd, nsy = abi.obs_output_sizes(o)
            m = [z(ndm), z(nfd), z(nsy), z(nsy), z(nsy)]
            integ.write_grid_device(o, *m)
            ref.append(m)
        reqs = [sharded.requested(o) for o in passes]
        outs = [[[z(n) for n in abi.obs_output_sizes(o)[:2]] + [z(abi.obs_output_sizes(o)[2])
                                                                for _ in range(3)]
                 for o in passes] for _ in range(nshards)]
        fd = outs[0][0][1]                       # pass 0's FD output, shared by the shards
        for s in range(passes[0].total_shell):
            n = abi.npix(passes[0].nside_shell[s])
            parts = []
            for r in range(nshards):
                t = {"dm": z(n), "fd": z(n), "iqu": [[z(n) for _ in range(3)] for _ in passes]}
                integ.shell_integrate_multi_device(passes, s, r, nshards, fd, t["dm"], t["fd"],
                                                   t["iqu"])
                parts.append(t)
            fd_sum = sum(t["fd"] for t in parts)             # the per-shell all-reduce
            for r in range(nshards):
                for f, o in enumerate(passes):
                    rq = reqs[f]
                    tmp = [parts[r]["dm"] if rq["dm"] else None, fd_sum] + parts[r]["iqu"][f]
                    out = list(outs[r][f])
                    if rq["fd"]:
                        out[1] = fd if r == 0 else z(len(fd))   # one FD output for all
                    integ.shell_merge_device(o, s, tmp, [out[j] if rq[k] else None
                                                         for j, k in enumerate(sharded.MAPS)])
        integ.sync()
        for f, o in enumerate(passes):
            for j, k in enumerate(sharded.MAPS):
                if not reqs[f][k]:
                    continue
                got = fd if k == "fd" else sum(outs[r][f][j] for r in range(nshards))
                e = rel_err(got.cpu().numpy(), ref[f][j].cpu().numpy())
                assert e <= 1e-5, (f, k, e)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_pass_end_merge_matches_per_shell_merges_bit_for_bit(fields32, precision):
    """hxg_write_grid_device and hxg_write_grid_multi keep every shell's DM
    and Stokes maps and merge them once at the end of the pass; the public
    per-shell calls (one shard) merge after each shell.  Both add the same
    shell values in the same order into zeroed outputs, so the maps agree
    exactly: pass by pass (the one-pass kernel in both) and for the
    Pipeline's three passes (fused in both in the FP32C form), with the
    interpolation tables and without them."""
    from hammurabix_b200.integrator import Integrator
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev) if n else None
    maps = lambda o: [z(n) for n in abi.obs_output_sizes(o)[:2]] + \
        [z(abi.obs_output_sizes(o)[2]) for _ in range(3)]
    # shells below and at the output Nside 32
    passes = W.frequency_passes(W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=0.408),
                                [0.408, 1.4, 30.0])
    nmax = abi.npix(32)
    with Integrator(precision) as integ:
        integ.set_stream(stream.cuda_stream)
        integ.set_models(W.grid_models())
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        whole = [maps(o) for o in passes]
        integ.write_grid_multi_device(list(zip(passes, whole)))
        per = [dict(zip(sharded.MAPS, maps(o))) for o in passes]
        sharded.write_passes_sharded(integ, passes, per, sharded.make_shell_maps(nmax, z), 0, 1,
                                     lambda t: None)
        single, single_per = [], []
        for o in passes:
            m = maps(o)
            integ.write_grid_device(o, *m)
            single.append(m)
            p = dict(zip(sharded.MAPS, maps(o)))
            sharded.write_grid_sharded(integ, o, p, {k: z(nmax) for k in sharded.MAPS}, 0, 1,
                                       lambda t: None)
            single_per.append(p)
        integ.sync()
    # no interpolation tables: the merges find the weights in place
    with Integrator(precision) as integ:
        integ.set_stream(stream.cuda_stream)
        integ.set_interp_cache(0)
        integ.set_models(W.grid_models())
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        notab = [maps(o) for o in passes]
        integ.write_grid_multi_device(list(zip(passes, notab)))
        integ.sync()
    for f, o in enumerate(passes):
        req = sharded.requested(o)
        for j, k in enumerate(sharded.MAPS):
            if not req[k]:
                continue
            a = per[f][k].cpu().numpy()
            assert np.abs(a).max() > 0, (f, k)
            assert np.array_equal(whole[f][j].cpu().numpy(), a), (f, k, "passes")
            assert np.array_equal(notab[f][j].cpu().numpy(), a), (f, k, "no tables")
            assert np.array_equal(single[f][j].cpu().numpy(),
                                  single_per[f][k].cpu().numpy()), (f, k, "one pass")


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-5)])
@pytest.mark.parametrize("nshards", [2, 3])
def test_emulated_sharded_adjoint_matches_the_unsplit_adjoint(precision, tol, nshards):
    """The sharded adjoint (hxg_adjoint_shard_*) with the shards emulated one
    after another on one GPU, one handle per shard as one per GPU: the
    per-shell forward with its FD exchange and checkpoints, then the
    reverse pass with the per-shell sum of the shards' FD-map gradient
    terms; the shards' gradients summed (the all-reduce) against
    hxg_adjoint_device on one handle.  Spiral B + exponential n_e disk +
    CRE_ana with B and n_e random grids, 0.408 GHz with DM and FD (inner-
    shell Faraday rotation), random dL/d(maps)."""
    from hammurabix_b200.integrator import Integrator
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    n = 16
    obs = W.make_obs([4, 8, 16], 24.0, 0.1, freq_ghz=0.408)
    m = W.spiral_models()
    m.brnd = abi.HXG_BRND_GRID
    m.ternd = abi.HXG_TERND_GRID
    desc = W.grid_desc(n)
    rng = np.random.Generator(np.random.PCG64(21))
    b = [torch.tensor(rng.standard_normal(n ** 3) * 0.5e-6, device=dev) for _ in range(3)]
    ne = torch.tensor(0.01 * rng.standard_normal(n ** 3), device=dev)
    z = lambda k: torch.zeros(k, dtype=torch.float64, device=dev)
    ndm, nfd, nsy = abi.obs_output_sizes(obs)
    g = {k: torch.tensor(rng.standard_normal(c), device=dev)
         for k, c in zip(sharded.MAPS, (ndm, nfd, nsy, nsy, nsy))}

    def handle():
        ig = Integrator(precision)
        ig.set_stream(stream.cuda_stream)
        ig.set_models(m)
        ig.upload_grid_device(abi.HXG_FIELD_BRND, desc, b)
        ig.upload_grid_device(abi.HXG_FIELD_TERND, desc, [ne])
        ig.set_checkpointing(True)
        return ig

    def grads():
        return {"params": z(abi.HXG_NUM_PARAMS), "b": [z(n ** 3) for _ in range(3)],
                "ne": z(n ** 3)}

    ref = handle()
    ref.write_grid_device(obs, z(ndm), z(nfd), z(nsy), z(nsy), z(nsy))
    rg = grads()
    ref.adjoint_device(obs, *[g[k] for k in sharded.MAPS], grad_params=rg["params"],
                       grad_b=rg["b"], grad_ne=rg["ne"])
    igs = [handle() for _ in range(nshards)]
    # forward: per shell, every shard's shell maps, their sum (the all-reduce
    # of the FD map) merged into the FD output every shard reads
    fd = z(nfd)
    nmax = abi.npix(max(obs.nside_shell[s] for s in range(obs.total_shell)))
    for s in range(obs.total_shell):
        ns = abi.npix(obs.nside_shell[s])
        parts = []
        for r, ig in enumerate(igs):
            t = [z(nmax)[:ns] for _ in sharded.MAPS]
            ig.shell_integrate_device(obs, s, r, nshards, fd, t)
            parts.append(t)
        tsum = [sum(p[j] for p in parts) for j in range(5)]
        igs[0].shell_merge_device(obs, s, tsum, [z(ndm), fd, z(nsy), z(nsy), z(nsy)])
    # reverse pass
    for r, ig in enumerate(igs):
        ig.adjoint_shard_begin(obs, r, nshards)
    gfd = g["fd"].clone()
    for s in reversed(range(obs.total_shell)):
        incs = [z(nfd) for _ in igs]
        for ig, inc in zip(igs, incs):
            ig.adjoint_shard_shell(obs, s, g["dm"], gfd, g["is"], g["qs"], g["us"], inc)
        gfd += sum(incs)
    tot = grads()
    for ig in igs:
        part = grads()
        ig.adjoint_shard_finish(part["params"], part["b"], part["ne"])
        tot["params"] += part["params"]
        tot["ne"] += part["ne"]
        for k in range(3):
            tot["b"][k] += part["b"][k]
    torch.cuda.synchronize()
    pairs = [("params", tot["params"], rg["params"]), ("ne", tot["ne"], rg["ne"])] + \
        [(f"b{k}", tot["b"][k], rg["b"][k]) for k in range(3)]
    for name, a, r in pairs:
        a, r = a.cpu().numpy(), r.cpu().numpy()
        assert np.abs(r).max() > 0, name
        assert rel_err(a, r) <= tol, (name, rel_err(a, r))
    # parameters one by one (their scales differ by orders of magnitude; the
    # FP32C shards split rays over other lane counts than the unsplit pass)
    a, r = tot["params"].cpu().numpy(), rg["params"].cpu().numpy()
    ptol = tol if precision == "fp64" else 1e-4
    for k in range(abi.HXG_NUM_PARAMS):
        assert abs(a[k] - r[k]) <= ptol * abs(r[k]) + 1e-300, (k, a[k], r[k])
    # one reverse pass per forward pass; a finish without a begin is refused
    from hammurabix_b200._lib import HxgError
    with pytest.raises(HxgError) as e:
        igs[0].adjoint_shard_begin(obs, 0, nshards)
    assert e.value.status == abi.HXG_ERR_STATE
    with pytest.raises(HxgError):
        igs[0].adjoint_shard_finish(z(abi.HXG_NUM_PARAMS))
    # the whole-pass forward leaves no per-shell checkpoints
    with pytest.raises(HxgError):
        ref.adjoint_shard_begin(obs, 0, 1)
    for ig in [ref] + igs:
        ig.close()
