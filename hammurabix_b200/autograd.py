"""PyTorch autograd for the line-of-sight integrator (FP64 or FP32C form).

``LOSMaps`` maps differentiable inputs -- the 8 regular-field parameters
(spiral B: b0, pitch, r_scale, h_scale; exponential n_e disk: n0, r_scale,
h_scale; CRE j0, all in CGS as in include/hxg.h) and the B and n_e grid
values -- to the DM / FD / I / Q / U maps of one frequency pass.  Its
backward runs the adjoint kernel (hxg_adjoint_device): one backward sweep
per shell from the forward pass's per-shell checkpoints.

    maps = LOSMaps(obs, base_models, grid_desc)
    dm, fd, i, q, u = maps(params, b_grid, ne_grid)   # params: (8,) float64
    loss = ((q - q_target) ** 2).sum(); loss.backward()

The B grid is read as the random-field slot (Grid_brnd) and the n_e grid as
the random n_e slot (Grid_ternd) on top of the analytic models.
"""
import torch

from . import abi
from .integrator import Integrator

PARAM_NAMES = ("b0", "pitch", "r_scale_B", "h_scale_B", "n0", "r_scale_n", "h_scale_n", "j0")


def apply_params(models, params):
    """Copy the 8 parameters (host floats) into an abi.Models."""
    m = abi.Models.from_buffer_copy(models)
    p = [float(v) for v in params]
    m.spiral.b0, m.spiral.pitch, m.spiral.r_scale, m.spiral.h_scale = p[0:4]
    m.te_exp.n0, m.te_exp.r_scale, m.te_exp.h_scale = p[4:7]
    if m.cre == abi.HXG_CRE_ANA:
        m.cre_ana.j0 = p[7]
    else:
        m.cre_unif.j0 = p[7]
    return m


def params_of(models):
    m = models
    j0 = m.cre_ana.j0 if m.cre == abi.HXG_CRE_ANA else m.cre_unif.j0
    return [m.spiral.b0, m.spiral.pitch, m.spiral.r_scale, m.spiral.h_scale,
            m.te_exp.n0, m.te_exp.r_scale, m.te_exp.h_scale, j0]


class _LOSFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, bx, by, bz, ne, session):
        s = session
        m = apply_params(s.base, params.detach().cpu().tolist())
        s.integ.set_models(m)
        s.integ.upload_grid_device(abi.HXG_FIELD_BRND, s.desc,
                                   [bx.detach().contiguous(), by.detach().contiguous(),
                                    bz.detach().contiguous()])
        s.integ.upload_grid_device(abi.HXG_FIELD_TERND, s.desc, [ne.detach().contiguous()])
        outs = s.new_outputs()
        s.integ.write_grid_device(s.obs, outs[0], outs[1], outs[2], outs[3], outs[4])
        s.integ.sync()
        ctx.session = s
        return tuple(o if o is not None else torch.zeros(0, dtype=torch.float64,
                                                         device=s.device) for o in outs)

    @staticmethod
    def backward(ctx, g_dm, g_fd, g_is, g_qs, g_us):
        s = ctx.session
        dev = s.device
        n = s.desc.nx * s.desc.ny * s.desc.nz
        gpar = torch.zeros(abi.HXG_NUM_PARAMS,
                           dtype=torch.float64, device=dev)
        gb = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(3)]
        gne = torch.zeros(n, dtype=torch.float64, device=dev)
        ok = lambda g: g.contiguous() if (g is not None and g.numel() > 0) else None
        s.integ.adjoint_device(s.obs, ok(g_dm), ok(g_fd), ok(g_is), ok(g_qs), ok(g_us),
                               gpar, gb, gne)
        return gpar, gb[0], gb[1], gb[2], gne, None


class LOSMaps:
    """Differentiable forward map of one frequency pass.  precision "fp64"
    (the parity form, every model) or "fp32c" (the FP32-compensated forward
    and its adjoint: the grid workloads' models -- spiral B, exponential n_e
    disk, CRE_ana with a constant index -- on one grid geometry)."""

    def __init__(self, obs, base_models, grid_desc, device=0, precision="fp64"):
        self.obs = obs
        self.base = abi.Models.from_buffer_copy(base_models)
        self.base.brnd = abi.HXG_BRND_GRID
        self.base.ternd = abi.HXG_TERND_GRID
        self.desc = grid_desc
        self.device = torch.device("cuda", device)
        self.precision = precision
        self.integ = Integrator(precision, device=device)
        self.integ.set_checkpointing(True)

    def new_outputs(self):
        ndm, nfd, nsy = abi.obs_output_sizes(self.obs)
        mk = lambda k: torch.zeros(k, dtype=torch.float64, device=self.device) if k else None
        return [mk(ndm), mk(nfd), mk(nsy), mk(nsy), mk(nsy)]

    def __call__(self, params, b_grid, ne_grid):
        bx, by, bz = b_grid
        return _LOSFunction.apply(params, bx, by, bz, ne_grid, self)
