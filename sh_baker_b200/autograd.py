"""torch.autograd wrapper of the differentiable bake: forward = shb_bake with
the given material albedos and light intensities set on the scene
(shb_scene_set_params), backward = the path-replay adjoint (shb_backward)
over the same G-buffer, config and random stream."""
from __future__ import annotations

import torch

from . import api


class SHBake(torch.autograd.Function):
    """sh = SHBake.apply(albedo, light_intensity, bake).

    albedo: (materials, 3) linear base colours, light_intensity: (lights,);
    bake: an api.BatchBake.  Returns the SH9 lightmap of the supersampled
    G-buffer as a CUDA float32 tensor (W*s*H*s, 9, 3).  Gradients flow to
    albedo and light_intensity (float32, on their own devices)."""

    @staticmethod
    def forward(ctx, albedo, light_intensity, bake):
        bake.scene.set_params(albedo.detach().cpu().numpy(), light_intensity.detach().cpu().numpy())
        n = bake.gbuffer.width * bake.gbuffer.height
        sh = torch.empty(n * 27, dtype=torch.float32, device="cuda")
        env = torch.empty(n, dtype=torch.float32, device="cuda")
        torch.cuda.current_stream().synchronize()
        api.bake_plain_device(bake, sh, env)
        ctx.bake = bake
        ctx.params = (albedo.detach().cpu().numpy().copy(), light_intensity.detach().cpu().numpy().copy())
        ctx.devices = (albedo.device, light_intensity.device)
        return sh.view(n, 9, 3)

    @staticmethod
    def backward(ctx, grad_sh):
        bake = ctx.bake
        # the scene may have been re-parameterised since the forward
        bake.scene.set_params(*ctx.params)
        g = grad_sh.detach().to(device="cuda", dtype=torch.float32).contiguous().view(-1)
        torch.cuda.current_stream().synchronize()
        d_alb, d_li = api.Backward(bake, g)
        return (torch.as_tensor(d_alb, dtype=torch.float32, device=ctx.devices[0]),
                torch.as_tensor(d_li, dtype=torch.float32, device=ctx.devices[1]), None)


def bake_sh(albedo: torch.Tensor, light_intensity: torch.Tensor, bake: api.BatchBake) -> torch.Tensor:
    return SHBake.apply(albedo, light_intensity, bake)
