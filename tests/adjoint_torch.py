"""Test-side torch.autograd.Function around frt_adjoint (the gradient harness only): the inputs
are per-source luminosity factors and per-cell density factors of one box, the output is the
adjoint's objective J (FP64, computed on the device), and backward returns the adjoint's
gradients scaled to those factors."""
import numpy as np
import torch

from flexrt_imaging_reion_b200 import rt, workloads as W


class GammaSubboxObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lum_scale, nh_scale, spec, seed, lo, hi):
        inp = W.make_inputs(spec)
        # factors per gridded source (frt_set_sources order): every catalogue source of a cell
        # takes its cell's factor
        ijk, _ = W.grid_sources(inp)
        n = spec.n
        gidx = {int((i * n + j) * n + k): q for q, (i, j, k) in enumerate(ijk.tolist())}
        lx0 = float(spec.lx0_kpc())
        idx = np.floor(inp.src_pos / W.HH / lx0 * 1e3 * n).astype(np.int64) % n
        flat = (idx[:, 0] * n + idx[:, 1]) * n + idx[:, 2]
        f = lum_scale.detach().cpu().numpy()
        inp.src_lum = inp.src_lum * np.array([f[gidx[int(c)]] for c in flat])
        sc = nh_scale.detach().cpu().numpy().reshape(inp.delta1.shape)
        inp.delta1 = (inp.delta1.astype(np.float64) * sc).astype(np.float32)
        with rt.RTContext([inp], [seed], ray_capacity=1 << 20) as c:
            c.setup()
            J, dl, dnh = c.adjoint(lo, hi)
            nh = c.get_field(0, "NH").astype(np.float64)
            _, lums = W.grid_sources(inp)
        # chain rule to the factors: dJ/dlam_s = dJ/dL_s L_s, dJ/dsc_c = dJ/dnH_c nH_c
        g_l = torch.tensor(dl * lums, dtype=torch.float64)
        g_s = torch.tensor(dnh.astype(np.float64) * nh, dtype=torch.float64)
        ctx.save_for_backward(g_l, g_s)
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        g_l, g_s = ctx.saved_tensors
        return grad_out * g_l, grad_out * g_s, None, None, None, None
