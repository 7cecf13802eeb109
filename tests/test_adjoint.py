"""Adjoint (hxg_adjoint_device through torch.autograd) against central finite
differences of the FP64 forward, on a reduced config-4 workload: analytic
spiral B + exponential n_e disk + CRE_ana, a random B grid (Grid_brnd) and a
random n_e grid (Grid_ternd), three shells, DM + FD + sync with inner-shell
Faraday rotation.

Loss: sum over I, Q, U, FD, DM of w_k (map_k - target_k)^2 / sigma_k^2 with
targets from 1%-perturbed parameters.  Finite differences: central
differences with steps h and h/2 combined by Richardson extrapolation (error
O(h^4): at 0.408 GHz the Faraday phase makes the loss strongly nonlinear),
h = 1e-4 relative for parameters and 1e-4 of the grid rms for voxels.
"""
import numpy as np
import pytest

from hammurabix_b200 import abi, units as U, workloads as W

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _setup(freq_ghz):
    from hammurabix_b200.autograd import LOSMaps, params_of
    n = 16
    obs = W.make_obs([4, 8, 16], 24.0, 0.1, freq_ghz=freq_ghz)
    base = W.spiral_models()
    base.tereg = abi.HXG_TEREG_EXPDISK
    desc = W.grid_desc(n)
    rng = np.random.Generator(np.random.PCG64(21))
    dev = torch.device("cuda", 0)
    b = [torch.tensor(rng.standard_normal(n ** 3) * 0.5e-6, dtype=torch.float64, device=dev)
         for _ in range(3)]
    ne = torch.tensor(0.01 * rng.standard_normal(n ** 3), dtype=torch.float64, device=dev)
    maps = LOSMaps(obs, base, desc)
    p0 = torch.tensor(params_of(maps.base), dtype=torch.float64, device=dev)
    return maps, p0, b, ne


def _loss_fn(maps, targets, weights):
    def loss(p, b, ne):
        outs = maps(p, b, ne)
        tot = 0.
        for o, t, w in zip(outs, targets, weights):
            if o.numel():
                tot = tot + (w * (o - t) ** 2).sum()
        return tot
    return loss


def _richardson(f, x0, h):
    """Central difference of f at x0 along a unit step, Richardson-extrapolated
    from steps h and h/2."""
    def cd(s):
        return (f(x0 + s) - f(x0 - s)) / (2 * s)
    return (4.0 * cd(0.5 * h) - cd(h)) / 3.0


def _targets(maps, p0, b, ne):
    with torch.no_grad():
        pert = p0 * (1.0 + 0.01 * torch.tensor([1, -1, 1, 1, -1, 1, -1, 1], dtype=torch.float64,
                                                device=p0.device))
        outs = maps(pert, b, ne)
    weights = []
    for o in outs:
        s = o.abs().max().item() if o.numel() else 1.0
        weights.append(1.0 / (0.01 * s) ** 2 if s > 0 else 0.0)
    return [o.clone() for o in outs], weights


@pytest.mark.parametrize("freq", [23.0, 0.408])
def test_adjoint_matches_finite_differences(freq):
    maps, p0, b, ne = _setup(freq)
    targets, weights = _targets(maps, p0, b, ne)
    loss = _loss_fn(maps, targets, weights)
    p = p0.clone().requires_grad_(True)
    bb = [t.clone().requires_grad_(True) for t in b]
    nn = ne.clone().requires_grad_(True)
    L = loss(p, bb, nn)
    L.backward()
    gp = p.grad.cpu().numpy()
    # parameters
    for k in range(8):
        def f_par(x, k=k):
            pk = p0.clone()
            pk[k] = x
            with torch.no_grad():
                return loss(pk, b, ne).item()
        fd = _richardson(f_par, p0[k].item(), 1e-4 * abs(p0[k].item()))
        scale = max(abs(fd), abs(gp[k]), 1e-30)
        assert abs(gp[k] - fd) <= 2e-4 * scale + 1e-12 * abs(L.item()) / abs(p0[k].item()), \
            (k, gp[k], fd)
    # random voxels of the B and n_e grids
    rng = np.random.Generator(np.random.PCG64(6))
    grads = [t.grad for t in bb] + [nn.grad]
    arrays = list(b) + [ne]
    checked = 0
    for comp in range(4):
        g = grads[comp]
        # probe the voxels with the largest gradients plus random ones
        idx = list(torch.topk(g.abs(), 4).indices.cpu().numpy()) + \
            list(rng.integers(0, g.numel(), 4))
        rms = arrays[comp].std().item()
        for i in idx:
            def f_vox(x, comp=comp, i=i):
                a = [t.clone() for t in arrays]
                a[comp][i] = x
                with torch.no_grad():
                    return loss(p0, a[:3], a[3]).item()
            fd = _richardson(f_vox, arrays[comp][i].item(), 1e-4 * rms)
            an = g[i].item()
            scale = max(abs(fd), abs(an))
            if scale == 0:
                continue
            assert abs(an - fd) <= 2e-4 * scale + 1e-9 * abs(g).max().item(), \
                (comp, int(i), an, fd)
            checked += 1
    assert checked >= 16


def test_adjoint_cost_and_state_errors():
    maps, p0, b, ne = _setup(1.4)
    from hammurabix_b200 import _lib
    integ = maps.integ
    with pytest.raises(_lib.HxgError) as e:
        integ.adjoint_device(maps.obs)     # no checkpointed forward yet
    assert e.value.status == abi.HXG_ERR_STATE


@pytest.mark.slow
def test_adjoint_config4_full_size():
    """Config 4 as stated: 256^3 B (Grid_brnd) and n_e (Grid_ternd) grids
    of the seeded synthetic fields, Nside 64/128/256 over 3 shells to 30 kpc
    at 0.01 kpc, one 23 GHz pass with DM and FD; loss = sum over I, Q, U and
    FD of ((map - target) / sigma)^2 with the target made from the 8
    parameters perturbed by 1 % plus Gaussian noise of sigma = 1 % of each
    map's maximum (seed 5).  The adjoint gradient is checked against central
    differences (step 1e-4 relative, Richardson-extrapolated) for all 8
    parameters and 32 voxels drawn with seed 6 among those the rays reach
    (nonzero gradient): 16 of B (the three components) and 16 of n_e.  The
    difference of two losses is summed from the difference of their maps,
    which is exactly zero on pixels the perturbation does not reach, so a
    single voxel's effect is not lost in the rounding of the 3-million-pixel
    sum."""
    from hammurabix_b200.autograd import LOSMaps, params_of
    dev = torch.device("cuda", 0)
    n = 256
    bx, by, bz, ne = W.random_grids_torch(n, 1, 2, device=dev)
    b = [t.double().reshape(-1).contiguous() for t in (bx, by, bz)]
    dne = (ne.double().reshape(-1) - 0.03).contiguous()   # fluctuation on the disk
    del bx, by, bz, ne
    base = W.spiral_models()
    base.tereg = abi.HXG_TEREG_EXPDISK
    obs = W.make_obs([64, 128, 256], 30.0, 0.01, freq_ghz=23.0)
    maps = LOSMaps(obs, base, W.grid_desc(n))
    p0 = torch.tensor(params_of(maps.base), dtype=torch.float64, device=dev)
    keep = (1, 2, 3, 4)          # FD, I, Q, U (dm, fd, is, qs, us order)
    gen = torch.Generator(device=dev).manual_seed(5)
    with torch.no_grad():
        sign = torch.tensor([1, -1, 1, 1, -1, 1, -1, 1], dtype=torch.float64, device=dev)
        outs = maps(p0 * (1.0 + 0.01 * sign), b, dne)
        sig = {k: 0.01 * outs[k].abs().max().item() for k in keep}
        target = {k: outs[k] + sig[k] * torch.randn(outs[k].shape, generator=gen,
                                                     dtype=torch.float64, device=dev)
                  for k in keep}

    def loss_of(o):
        return sum((((o[k] - target[k]) / sig[k]) ** 2).sum() for k in keep)

    def dloss(op, om):
        """loss(op) - loss(om) from the map differences."""
        return sum(((op[k] - om[k]) * (op[k] + om[k] - 2.0 * target[k])).sum().item()
                   / sig[k] ** 2 for k in keep)

    p = p0.clone().requires_grad_(True)
    bb = [t.clone().requires_grad_(True) for t in b]
    nn = dne.clone().requires_grad_(True)
    L = loss_of(maps(p, bb, nn))
    L.backward()

    def fwd(pv, bv, nv):
        with torch.no_grad():
            return [t.clone() for t in maps(pv, bv, nv)]

    def richardson(make, h):
        def cd(s):
            return dloss(make(s), make(-s)) / (2.0 * s)
        return (4.0 * cd(0.5 * h) - cd(h)) / 3.0

    gp = p.grad.cpu().numpy()
    for k in range(8):
        h = 1e-4 * abs(p0[k].item())

        def make(s, k=k):
            q = p0.clone()
            q[k] += s
            return fwd(q, b, dne)
        fd = richardson(make, h)
        assert abs(gp[k] - fd) <= 2e-4 * max(abs(fd), abs(gp[k])) + 1e-10 * abs(L.item()) / abs(
            p0[k].item()), (k, gp[k], fd)
    rng = np.random.Generator(np.random.PCG64(6))
    grads = [t.grad for t in bb] + [nn.grad]
    arrays = list(b) + [dne]
    checked = 0
    for comp, count in ((0, 6), (1, 5), (2, 5), (3, 16)):
        g = grads[comp]
        reach = torch.nonzero(g.abs() > 1e-6 * g.abs().max()).reshape(-1).cpu().numpy()
        rms = arrays[comp].std().item()
        for i in rng.choice(reach, size=count, replace=False):
            def make(s, comp=comp, i=i):
                a = [t.clone() for t in arrays]
                a[comp][i] += s
                return fwd(p0, a[:3], a[3])
            fd = richardson(make, 1e-4 * rms)
            an = g[i].item()
            assert abs(an - fd) <= 2e-4 * max(abs(fd), abs(an)) + 1e-8 * g.abs().max().item(), \
                (comp, int(i), an, fd)
            checked += 1
    assert checked == 32


def _grads(precision, freq, n=16, nsides=(4, 8, 16), r_max=24.0, res=0.1, seed=21):
    """Loss gradients (parameters, B grid, n_e grid) of the adjoint in the
    given form, on the reduced config-4 setup with a seeded target."""
    from hammurabix_b200.autograd import LOSMaps, params_of
    obs = W.make_obs(list(nsides), r_max, res, freq_ghz=freq)
    base = W.spiral_models()
    base.tereg = abi.HXG_TEREG_EXPDISK
    dev = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(seed))
    b = [torch.tensor(rng.standard_normal(n ** 3) * 0.5e-6, dtype=torch.float64, device=dev)
         for _ in range(3)]
    ne = torch.tensor(0.01 * rng.standard_normal(n ** 3), dtype=torch.float64, device=dev)
    # the same targets for both forms: made by the FP64 form
    ref = LOSMaps(obs, base, W.grid_desc(n), precision="fp64")
    p0 = torch.tensor(params_of(ref.base), dtype=torch.float64, device=dev)
    targets, weights = _targets(ref, p0, b, ne)
    maps = ref if precision == "fp64" else LOSMaps(obs, base, W.grid_desc(n), precision=precision)
    p = p0.clone().requires_grad_(True)
    bb = [t.clone().requires_grad_(True) for t in b]
    nn = ne.clone().requires_grad_(True)
    _loss_fn(maps, targets, weights)(p, bb, nn).backward()
    return p.grad.cpu().numpy(), [t.grad.cpu().numpy() for t in bb], nn.grad.cpu().numpy()


@pytest.mark.parametrize("freq", [23.0, 0.408])
def test_fp32c_adjoint_matches_fp64_gradient(freq):
    """The FP32C form's adjoint (hxg_adjoint32.cuh: FP32 fields and
    emissivity, FP64 Faraday path) against the FP64 GPU gradient on the same
    inputs and loss: every parameter gradient and the voxel gradients of the
    B and n_e grids agree to 1e-4 of their largest magnitude."""
    gp64, gb64, gn64 = _grads("fp64", freq)
    gp32, gb32, gn32 = _grads("fp32c", freq)
    scale = np.abs(gp64)
    for k in range(8):
        assert abs(gp32[k] - gp64[k]) <= 1e-4 * scale[k] + 1e-12 * scale.max(), \
            (k, gp32[k], gp64[k])
    for a, r in list(zip(gb32, gb64)) + [(gn32, gn64)]:
        assert np.abs(r).max() > 0
        e = np.abs(a - r).max() / np.abs(r).max()
        assert e <= 1e-4, e


@pytest.mark.slow
def test_fp32c_adjoint_config4_vs_fp64_gradient():
    """The FP32C adjoint at config-4 size (256^3 grids, Nside 64/128/256, 3
    shells to 30 kpc, 23 GHz with DM and FD, target with 1 % noise) against
    the FP64 GPU gradient of the same loss: parameter gradients within 1e-4
    of each, voxel gradients within 1e-4 of their largest magnitude."""
    from hammurabix_b200.autograd import LOSMaps, params_of
    dev = torch.device("cuda", 0)
    n = 256
    bx, by, bz, ne = W.random_grids_torch(n, 1, 2, device=dev)
    b = [t.double().reshape(-1).contiguous() for t in (bx, by, bz)]
    dne = (ne.double().reshape(-1) - 0.03).contiguous()
    del bx, by, bz, ne
    base = W.spiral_models()
    base.tereg = abi.HXG_TEREG_EXPDISK
    obs = W.make_obs([64, 128, 256], 30.0, 0.01, freq_ghz=23.0)
    keep = (1, 2, 3, 4)
    grads = {}
    target = sig = None
    for prec in ("fp64", "fp32c"):
        maps = LOSMaps(obs, base, W.grid_desc(n), precision=prec)
        p0 = torch.tensor(params_of(maps.base), dtype=torch.float64, device=dev)
        if target is None:
            gen = torch.Generator(device=dev).manual_seed(5)
            with torch.no_grad():
                sign = torch.tensor([1, -1, 1, 1, -1, 1, -1, 1], dtype=torch.float64,
                                    device=dev)
                outs = maps(p0 * (1.0 + 0.01 * sign), b, dne)
                sig = {k: 0.01 * outs[k].abs().max().item() for k in keep}
                target = {k: outs[k] + sig[k] * torch.randn(outs[k].shape, generator=gen,
                                                             dtype=torch.float64, device=dev)
                          for k in keep}
        p = p0.clone().requires_grad_(True)
        bb = [t.clone().requires_grad_(True) for t in b]
        nn = dne.clone().requires_grad_(True)
        outs = maps(p, bb, nn)
        sum((((outs[k] - target[k]) / sig[k]) ** 2).sum() for k in keep).backward()
        grads[prec] = (p.grad.cpu().numpy(), [t.grad for t in bb] + [nn.grad])
    gp64, gv64 = grads["fp64"]
    gp32, gv32 = grads["fp32c"]
    for k in range(8):
        assert abs(gp32[k] - gp64[k]) <= 1e-4 * abs(gp64[k]), (k, gp32[k], gp64[k])
    for a, r in zip(gv32, gv64):
        m = r.abs().max().item()
        assert m > 0
        e = (a - r).abs().max().item() / m
        assert e <= 1e-4, e
