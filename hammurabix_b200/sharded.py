"""One frequency pass split across the ranks of a process group by shell
pixels: the multi-GPU form of Integrator::write_grid
(source/integrator/integrator.cc:23-134).

The pixels of a shell are independent; the only exchange is the Faraday
depth of the inner shells, which every pixel of the next shell reads from the
accumulated FD map (integrator.cc:78-86).  So, per shell, each rank integrates
its shard of the shell's NESTED pixels (zero elsewhere), the shell FD maps
are summed over the ranks (an all-reduce of one map of 12 nside_shell^2
doubles; the shards are disjoint, so the sum is the full map), and every rank
merges the complete FD map into its FD output, which is then identical on
all ranks.  The DM and Stokes maps are merged from each rank's partial shell
maps (the merge is linear) and summed onto rank 0 once at the end of the
pass (a reduce, not an all-reduce: no rank but the first needs them), so
after a pass rank 0 holds every output map and the other ranks the FD map
and their own partial DM / I / Q / U.  Every rank issues the same
collectives in the same order.

The adjoint of such a pass (adjoint_sharded) runs each rank's pixels shell
by shell from the outermost, with the mirror exchange: the ranks sum their
terms of dL/d(accumulated FD map) after each shell, and all-reduce the grid
and parameter gradients at the end.
"""
from . import abi

MAPS = ("dm", "fd", "is", "qs", "us")


def requested(obs):
    """Which of MAPS the pass writes."""
    return {"dm": bool(obs.do_dm), "fd": bool(obs.do_fd), "is": bool(obs.do_sync),
            "qs": bool(obs.do_sync), "us": bool(obs.do_sync)}


def shell_maps_needed(obs):
    """Which shell maps the kernel writes (the FD shell map whenever FD or
    sync is on)."""
    r = requested(obs)
    r["fd"] = bool(obs.do_fd or obs.do_sync)
    return r


def write_grid_sharded(integ, obs, outs, tmp, rank, world, reduce_sum, reduce_root=None):
    """One pass on this rank.

    integ: an Integrator; its device calls are ordered with the caller's
    current torch stream, where the zeroing and the reductions run (giving
    it that stream with Integrator.set_stream saves the event waits);
    outs: dict of the pass outputs (device tensors, the requested ones);
    tmp: dict of shell-map buffers of 12 max(nside_shell)^2 doubles;
    reduce_sum(t): in-place sum of t over the ranks onto every rank, in
    stream order (the per-shell FD map);
    reduce_root(t): in-place sum of t over the ranks onto rank 0 (the DM
    and Stokes outputs at the end of the pass); reduce_sum if None."""
    reduce_root = reduce_root or reduce_sum
    req, need = requested(obs), shell_maps_needed(obs)
    for k in MAPS:
        if req[k]:
            outs[k].zero_()
    out_list = [outs[k] if req[k] else None for k in MAPS]
    for s in range(obs.total_shell):
        n = abi.npix(obs.nside_shell[s])
        views = [tmp[k][:n] if need[k] else None for k in MAPS]
        integ.shell_integrate_device(obs, s, rank, world, outs["fd"] if req["fd"] else None,
                                     views)
        if world > 1 and req["fd"]:
            reduce_sum(views[1])
        integ.shell_merge_device(obs, s, views, out_list)
    if world > 1:
        for k in ("dm", "is", "qs", "us"):
            if req[k]:
                reduce_root(outs[k])


def adjoint_sharded(integ, obs, g, grads, rank, world, reduce_sum, zeros):
    """The reverse pass of a pass that write_grid_sharded ran on this rank
    with checkpointing on (Integrator.set_checkpointing): the gradients of a
    scalar loss of the maps, the multi-GPU form of hxg_adjoint_device.

    Each rank runs the adjoint of its own pixels, shell by shell from the
    outermost.  The one exchange mirrors the forward's: every pixel of an
    inner shell read the accumulated FD map, so its gradient dL/d(FD map)
    collects terms from every pixel of the outer shells; after each shell
    the ranks sum their terms (reduce_sum) and add them to the map before
    the next shell.  At the end each rank holds its pixels' share of the
    grid and parameter gradients, summed over the ranks (reduce_sum: the
    grid-gradient all-reduce).

    g: dict of dL/d(outputs) keyed like MAPS (torch CUDA float64, None =
    zero); grads: dict "params" (HXG_NUM_PARAMS doubles), "b" (3 tensors or
    None), "ne" (tensor or None), filled with the full gradient on every
    rank; zeros(n): a zeroed float64 buffer of n elements on the device."""
    integ.adjoint_shard_begin(obs, rank, world)
    gfd = inc = None
    if obs.do_fd:
        n = abi.npix(obs.nside_fd)
        gfd = g["fd"].clone() if g.get("fd") is not None else zeros(n)
        inc = zeros(n)
    for s in reversed(range(obs.total_shell)):
        integ.adjoint_shard_shell(obs, s, g.get("dm"), gfd, g.get("is"), g.get("qs"),
                                  g.get("us"), inc)
        if inc is not None:
            if world > 1:
                reduce_sum(inc)
            gfd += inc
    integ.adjoint_shard_finish(grads.get("params"), grads.get("b"), grads.get("ne"))
    if world > 1:
        for t in [grads.get("params"), grads.get("ne")] + list(grads.get("b") or []):
            if t is not None:
                reduce_sum(t)


def make_shell_maps(n, zeros):
    """Shell-map buffers of n doubles for write_passes_sharded: the shared
    DM and FD maps and I/Q/U for up to three fused passes; zeros(n) makes
    one buffer."""
    return {"dm": zeros(n), "fd": zeros(n),
            "iqu": [[zeros(n) for _ in range(3)] for _ in range(3)]}


def _fused_group(integ, group, outs, tmp, rank, world, reduce_sum, reduce_root):
    """2 or 3 passes sharing one traversal per shell (the library refuses a
    group it cannot fuse before any work, with HXG_ERR_UNSUPPORTED)."""
    reqs = [requested(o) for o in group]
    first = True
    for s in range(group[0].total_shell):
        n = abi.npix(group[0].nside_shell[s])
        dm, fd = tmp["dm"][:n], tmp["fd"][:n]
        iqu = [[t[:n] for t in tmp["iqu"][f]] for f in range(len(group))]
        fd_out = next((outs[f]["fd"] for f, r in enumerate(reqs) if r["fd"]), None)
        if first:
            for f, r in enumerate(reqs):
                for k in MAPS:
                    if r[k]:
                        outs[f][k].zero_()
        integ.shell_integrate_multi_device(group, s, rank, world, fd_out, dm, fd, iqu)
        first = False
        if world > 1 and any(r["fd"] for r in reqs):
            reduce_sum(fd)
        for f, o in enumerate(group):
            r = reqs[f]
            integ.shell_merge_device(o, s, [dm if r["dm"] else None, fd] + iqu[f],
                                     [outs[f][k] if r[k] else None for k in MAPS])
    # every pass that writes FD merged the same complete maps: one FD output
    # was read by the kernels, the others are copies of it
    if world > 1:
        for f, r in enumerate(reqs):
            for k in ("dm", "is", "qs", "us"):
                if r[k]:
                    reduce_root(outs[f][k])


def write_passes_sharded(integ, passes, outs, tmp, rank, world, reduce_sum, reduce_root=None):
    """Several frequency passes (the Pipeline's order) on this rank: groups
    of up to three passes that the library can fuse share one traversal per
    shell (hxg_shell_integrate_multi_device); the others run one by one.
    outs: one dict of MAPS per pass; tmp: make_shell_maps(...); reduce_sum,
    reduce_root as in write_grid_sharded."""
    from ._lib import HxgError
    reduce_root = reduce_root or reduce_sum
    single = {"dm": tmp["dm"], "fd": tmp["fd"], "is": tmp["iqu"][0][0],
              "qs": tmp["iqu"][0][1], "us": tmp["iqu"][0][2]}
    k = 0
    while k < len(passes):
        done = False
        for nf in (3, 2):
            group = passes[k:k + nf]
            if len(group) < nf:
                continue
            try:
                _fused_group(integ, group, outs[k:k + nf], tmp, rank, world, reduce_sum,
                             reduce_root)
            except HxgError as e:
                if e.status != abi.HXG_ERR_UNSUPPORTED:
                    raise
                continue
            k += nf
            done = True
            break
        if not done:
            write_grid_sharded(integ, passes[k], outs[k], single, rank, world, reduce_sum,
                               reduce_root)
            k += 1
