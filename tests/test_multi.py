"""Several frequency passes at once (hxg_write_grid_multi): the FP32C form
runs up to three passes with the same geometry in one traversal per shell.
Every map must equal the map hxg_write_grid_device gives for that pass
alone; the arithmetic of each pass is the same, so the bar is 1e-6 of the
map maximum (a margin for the compiler's FMA contraction in the two kernel
instantiations), well inside the FP32C tolerance.  Cases: the Pipeline's
pass order (first pass with DM and FD, later ones synchrotron only, no
inner-shell Faraday rotation: Q2), a mask, a variable CRE index (per-pass
emissivity), a pass list of mixed geometry (split into fused groups and
single passes), and the FP64 form (passes one by one)."""
import numpy as np
import pytest

from conftest import rel_err
from hammurabix_b200 import abi, workloads as W

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-6


def _maps(o, dev):
    ndm, nfd, nsy = abi.obs_output_sizes(o)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev) if n else None
    return [z(ndm), z(nfd), z(nsy), z(nsy), z(nsy)]


def _integ(precision, fields32, models, dev, stream):
    from hammurabix_b200.integrator import Integrator
    ig = Integrator(precision)
    ig.set_stream(stream.cuda_stream)
    ig.set_models(models)
    bx, by, bz, ne = (torch.tensor(np.asarray(a, dtype=np.float64).reshape(-1), device=dev)
                      for a in fields32)
    ig.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(32), [bx, by, bz])
    ig.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(32), [ne])
    return ig


def _compare(ig, passes, dev):
    fused = [(o, _maps(o, dev)) for o in passes]
    ig.write_grid_multi_device(fused)
    single = []
    for o in passes:
        m = _maps(o, dev)
        ig.write_grid_device(o, *m)
        single.append(m)
    ig.sync()
    for k, ((o, a), b) in enumerate(zip(fused, single)):
        for j, name in enumerate(("dm", "fd", "I", "Q", "U")):
            if b[j] is None:
                continue
            x, y = a[j].cpu().numpy(), b[j].cpu().numpy()
            assert np.abs(y).max() > 0 or name == "fd", (k, name)
            assert rel_err(x, y) <= TOL, (k, name, rel_err(x, y))


@pytest.fixture
def dev_stream():
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    return dev, stream


@pytest.mark.parametrize("mask", [False, True])
def test_pipeline_pass_order(fields32, dev_stream, mask):
    dev, stream = dev_stream
    ig = _integ("fp32c", fields32, W.grid_models(), dev, stream)
    tmpl = W.make_obs([8, 16, 32], 20.0, 0.05, freq_ghz=0.408)
    passes = W.frequency_passes(tmpl, [0.408, 1.4, 30.0])
    if mask:
        rng = np.random.Generator(np.random.PCG64(3))
        ig.set_mask(16, (rng.random(abi.npix(16)) > 0.3).astype(np.float64))
        for o in passes:
            o.do_mask = 1
    assert passes[0].do_fd and not passes[1].do_fd
    _compare(ig, passes, dev)
    ig.close()


def test_variable_cre_index(fields32, dev_stream):
    dev, stream = dev_stream
    m = W.grid_models()
    m.cre_ana.beta = 0.02        # index varies with r: per-pass emissivity
    ig = _integ("fp32c", fields32, m, dev, stream)
    tmpl = W.make_obs([8, 16], 20.0, 0.05, freq_ghz=1.4)
    _compare(ig, W.frequency_passes(tmpl, [1.4, 5.0, 23.0]), dev)
    ig.close()


def test_mixed_geometry_and_fp64(fields32, dev_stream):
    dev, stream = dev_stream
    a = W.frequency_passes(W.make_obs([8, 16], 20.0, 0.05, freq_ghz=1.4), [1.4, 23.0])
    b = W.frequency_passes(W.make_obs([8, 16, 32], 18.0, 0.1, freq_ghz=0.408),
                           [0.408, 1.4, 30.0, 70.0])
    passes = a + b                # fused 2, then fused 3 + a single pass
    for prec in ("fp32c", "fp64"):
        ig = _integ(prec, fields32, W.grid_models(), dev, stream)
        _compare(ig, passes, dev)
        ig.close()


def test_passes_with_their_own_output_nsides(fields32, dev_stream):
    """One fused group whose passes write maps at different Nsides (the
    drop-in test's XML has 0.408 GHz at Nside 16 and 23 GHz at Nside 8):
    the merges go out per output Nside."""
    dev, stream = dev_stream
    ig = _integ("fp32c", fields32, W.grid_models(), dev, stream)
    tmpl = W.make_obs([4, 8, 16], 20.0, 0.05, freq_ghz=0.408, nside_out=16)
    passes = W.frequency_passes(tmpl, [0.408, 23.0, 5.0])
    passes[1].nside_sync = 8
    passes[2].nside_sync = 32
    _compare(ig, passes, dev)
    ig.close()
