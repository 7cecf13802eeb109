"""Batched forward (hxg_batch_create / hxg_batch_run): a batch of passes with
different spiral parameters, shell layouts, LOS lengths and frequencies,
run as one CUDA graph, against the same passes run one write_grid_device
call at a time on the same handle.  The batch may split pixels over a
different number of lanes than the single call, which changes the summation
order: FP64 agrees to the parity tolerance (1e-10), FP32C to 1e-5."""
import numpy as np
import pytest

from conftest import rel_err
from hammurabix_b200 import _lib, abi, units as U, workloads as W
from hammurabix_b200 import integrator as I

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _entries(rng, n):
    out = []
    for k in range(n):
        m = W.grid_models(W.spiral_models(b0_muG=rng.uniform(2, 8),
                                          pitch_deg=rng.uniform(-40, -5),
                                          hb_kpc=rng.uniform(0.5, 2)))
        nsh = int(rng.integers(1, 4))
        nsides = [8 * 2 ** s for s in range(nsh)]
        freq = [0.408, 1.4, 30.0][k % 3]
        o = W.make_obs(nsides, rng.uniform(15, 30), 0.05, freq_ghz=freq,
                       do_dm=(k % 3 == 0), do_fd=(k % 3 == 0))
        out.append((m, o))
    return out


def _outs(o, dev):
    ndm, nfd, nsy = abi.obs_output_sizes(o)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev) if n else None
    return {"dm": z(ndm), "fd": z(nfd), "is": z(nsy), "qs": z(nsy), "us": z(nsy)}


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32c", 1e-5)])
def test_batch_matches_per_entry_loop(fields32, precision, tol):
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(7))
    ents = _entries(rng, 9)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    with I.Integrator(precision) as integ:
        integ.set_models(ents[0][0])
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        ref = []
        for m, o in ents:
            integ.set_models(m)
            outs = _outs(o, dev)
            integ.write_grid_device(o, outs["dm"], outs["fd"], outs["is"], outs["qs"], outs["us"])
            ref.append(outs)
        integ.sync()
        got = [_outs(o, dev) for _, o in ents]
        b = integ.batch([(m, o, g) for (m, o), g in zip(ents, got)], tune=(precision == "fp32c"))
        for _ in range(2):      # a second run starts from zeroed outputs again
            b.run()
        integ.sync()
        info = b.info()
        b.close()
    assert info["samples"] > 0
    if precision == "fp32c":
        assert info["shapes_tried"] > 1 and info["best_ms"] > 0
    for k, (r, g) in enumerate(zip(ref, got)):
        for key, t in r.items():
            if t is None:
                continue
            e = rel_err(g[key].cpu().numpy(), t.cpu().numpy())
            assert e <= tol, (k, key, e)
            assert t.abs().max().item() > 0 or key == "fd"


def test_batch_rejects_mismatched_grid_reads_and_masks(fields32):
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(8))
    (m, o), = _entries(rng, 1)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    with I.Integrator("fp32c") as integ:
        integ.set_models(m)
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        other = abi.Models.from_buffer_copy(m)
        other.brnd = abi.HXG_BRND_NONE
        with pytest.raises(_lib.HxgError) as e:
            integ.batch([(other, o, _outs(o, dev))])
        assert e.value.status == abi.HXG_ERR_INVALID
        masked = abi.Obs.from_buffer_copy(o)
        masked.do_mask = 1
        with pytest.raises(_lib.HxgError) as e:
            integ.batch([(m, masked, _outs(o, dev))])
        assert e.value.status == abi.HXG_ERR_UNSUPPORTED


def test_batch_fuses_the_frequencies_of_a_parameter_set(fields32):
    """Consecutive entries with the same models and geometry (one parameter
    set at several frequencies, the first with DM and FD) share one
    traversal per shell in the FP32C batch; every entry's maps equal the
    pass run alone.  A lone entry and a pair sit between the groups."""
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(11))
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    ents = []
    for nf in (3, 1, 2, 3):
        m = W.grid_models(W.spiral_models(b0_muG=rng.uniform(2, 8),
                                          pitch_deg=rng.uniform(-40, -5)))
        nsides = [8 * 2 ** s for s in range(int(rng.integers(1, 4)))]
        rmax = rng.uniform(15, 30)
        for k, f in enumerate((30.0, 1.4, 0.408)[:nf]):
            ents.append((m, W.make_obs(nsides, rmax, 0.05, freq_ghz=f, do_dm=(k == 0),
                                       do_fd=(k == 0))))
    with I.Integrator("fp32c") as integ:
        integ.set_models(ents[0][0])
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        ref = []
        for m, o in ents:
            integ.set_models(m)
            outs = _outs(o, dev)
            integ.write_grid_device(o, outs["dm"], outs["fd"], outs["is"], outs["qs"], outs["us"])
            ref.append(outs)
        integ.sync()
        got = [_outs(o, dev) for _, o in ents]
        b = integ.batch([(m, o, g) for (m, o), g in zip(ents, got)], tune=True)
        b.run()
        integ.sync()
        info = b.info()
        b.close()
    assert info["samples"] == sum(W.samples_of(o) for _, o in ents)
    for k, (r, g) in enumerate(zip(ref, got)):
        for key, t in r.items():
            if t is None:
                continue
            e = rel_err(g[key].cpu().numpy(), t.cpu().numpy())
            assert e <= 1e-5, (k, key, e)
            assert t.abs().max().item() > 0 or key == "fd"


def test_batch_follows_new_grids_and_refuses_a_new_geometry(fields32):
    """Grids uploaded after hxg_batch_create with the same geometry are
    packed into the record arrays the graph reads: the next run gives the
    maps of the new grids.  A grid of another geometry moves the records,
    and the run is refused with HXG_ERR_STATE instead of reading them."""
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(12))
    ents = _entries(rng, 3)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    with I.Integrator("fp64") as integ:
        integ.set_models(ents[0][0])
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
        got = [_outs(o, dev) for _, o in ents]
        b = integ.batch([(m, o, g) for (m, o), g in zip(ents, got)])
        b.run()
        # new values, same geometry: half the field, twice the density (made
        # on torch's stream; the upload is ordered after them)
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32),
                                 [0.5 * bx, 0.5 * by, 0.5 * bz])
        integ.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [2.0 * ne])
        b.run()
        integ.sync()
        ref = []
        for m, o in ents:
            integ.set_models(m)
            outs = _outs(o, dev)
            integ.write_grid_device(o, outs["dm"], outs["fd"], outs["is"], outs["qs"], outs["us"])
            ref.append(outs)
        integ.sync()
        for k, (r, g) in enumerate(zip(ref, got)):
            for key, t in r.items():
                if t is None:
                    continue
                e = rel_err(g[key].cpu().numpy(), t.cpu().numpy())
                assert e <= 1e-10, (k, key, e)
        small = [t.reshape(32, 32, 32)[::2, ::2, ::2].contiguous().reshape(-1)
                 for t in (bx, by, bz)]
        integ.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(16), small)
        with pytest.raises(_lib.HxgError) as e:
            b.run()
        assert e.value.status == abi.HXG_ERR_STATE
        b.close()


def test_batch_config5_shape_against_oracle(oracle):
    """A config-5-shaped FP32C batch: 6 spiral parameter sets (b0, pitch,
    disk height drawn as in config 5) x 3 frequencies = 18 entries, 1-3
    shells of Nside 64/128/256 to 15-30 kpc at 0.01 kpc, one shared 64^3
    grid, in one graph with the autotuned shape.  Three entries (one of
    each shell count) are compared directly with the CPU oracle
    (oracle/hxo.c, the reference's write_grid restated) at the FP32C bound,
    and every entry with the per-pass loop."""
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(7))
    n = 64
    fields = W.random_grids(n, 5, 6)
    grids = W.grids_dict(n, *fields)
    ents, nsh_of = [], []
    for nsh in (3, 1, 2, 3, 2, 1):
        m = W.grid_models(W.spiral_models(b0_muG=rng.uniform(2, 8),
                                          pitch_deg=rng.uniform(-40, -5),
                                          hb_kpc=rng.uniform(0.5, 2)))
        rmax = rng.uniform(15, 30)
        for k, f in enumerate((30.0, 1.4, 0.408)):
            ents.append((m, W.make_obs([64 * 2 ** s for s in range(nsh)], rmax, 0.01,
                                       freq_ghz=f, do_dm=(k == 0), do_fd=(k == 0))))
            nsh_of.append(nsh)
    assert len(ents) >= 16
    dgrids = {f: (d, [torch.tensor(a, device=dev) for a in comps])
              for f, (d, comps) in grids.items()}
    with I.Integrator("fp32c") as integ:
        integ.set_models(ents[0][0])
        for f, (d, comps) in dgrids.items():
            integ.upload_grid_device(f, d, comps)
        got = [_outs(o, dev) for _, o in ents]
        b = integ.batch([(m, o, g) for (m, o), g in zip(ents, got)], tune=True)
        b.run()
        integ.sync()
        b.close()
        loop = []
        for m, o in ents:
            integ.set_models(m)
            outs = _outs(o, dev)
            integ.write_grid_device(o, outs["dm"], outs["fd"], outs["is"], outs["qs"], outs["us"])
            loop.append(outs)
        integ.sync()
    for k, (r, g) in enumerate(zip(loop, got)):
        for key, t in r.items():
            if t is not None:
                e = rel_err(g[key].cpu().numpy(), t.cpu().numpy())
                assert e <= 1e-5, (k, key, e)
    # one entry per shell count, the low frequency (strongest rotation) for
    # two of them and the DM/FD pass for the third
    picks = [nsh_of.index(1) + 2, nsh_of.index(2), nsh_of.index(3) + 2]
    for k in picks:
        m, o = ents[k]
        ref = oracle.write_grid(o, m, grids)
        for key in ("dm", "fd", "is", "qs", "us"):
            if ref[key] is None:
                continue
            assert np.abs(ref[key]).max() > 0, (k, key)
            e = rel_err(got[k][key].cpu().numpy(), ref[key])
            assert e <= 1e-5, (k, nsh_of[k], key, e)
