"""Differentiable spectral rendering: the film as a function of the material tables.

The reference renders forward only; this module adds gradients of an image
loss with respect to the spectral material parameters, computed by the
path-replay adjoint kernel of libspectral.so (ts_adjoint_pass):

    film = render_film(renderer, mat_f32, eem, first_pass, num_blocks)   # [B, H, W] float64
    xyz = film_to_xyz(film, cmf, renderer.cmf_scale)                      # [H, W, 3]
    loss = ((xyz - target) ** 2).sum()
    loss.backward()            # mat_f32.grad [M, 6, B], eem.grad [E, B, B]

Forward renders ``num_blocks`` whole spectral blocks (pass i renders band
i mod B with random stream first_pass + i) and returns the running mean over
blocks, as average_and_reset_block leaves it (main.py:1592-1607); it records
each path's total deposit (ts_record_paths).  Backward re-runs exactly those
paths from their random streams and accumulates the gradient in FP64; with the
forward's records it needs one replay per path, not two (a path that volume
fluorescence moved to another band is replayed twice).  Gradients exist for every table entry except the
refractive index (property 0), which is returned as zero.
"""
import torch


class _RenderFilm(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mat_f32, eem, renderer, first_pass, num_blocks):
        r = renderer
        mat = mat_f32.detach().to(r.device, torch.float32).contiguous()
        em = None if eem is None else eem.detach().to(r.device, torch.float32).contiguous()
        r.update_materials(mat, em)
        r.clear_pixel_space()
        B = r.config.bands
        # records let the adjoint skip its weight replay; only worth it when a gradient will follow
        r.record_paths(first_pass, num_blocks * B if any(ctx.needs_input_grad[:2]) else 0)
        for blk in range(num_blocks):
            r.cast_rays_bundle(0, B, pass_idx=first_pass + blk * B)  # one launch per block
            r.average_and_reset_block(blk + 1)
        film = r.mean_film.clone()
        ctx.renderer = r
        ctx.first_pass = first_pass
        ctx.num_blocks = num_blocks
        ctx.has_eem = eem is not None
        ctx.mat_dtype = mat_f32.dtype
        ctx.eem_dtype = None if eem is None else eem.dtype
        ctx.materials_version = r.materials_version
        ctx.save_for_backward(mat, em if em is not None else mat.new_empty(0))
        return film

    @staticmethod
    def backward(ctx, grad_film):
        r = ctx.renderer
        mat, em = ctx.saved_tensors
        # the adjoint replays the forward pass's paths: same tables, same streams
        # (re-uploaded only if they changed since, which also retires the records)
        if r.materials_version != ctx.materials_version:
            r.update_materials(mat, em if ctx.has_eem else None)
        adj = (grad_film.to(r.device, torch.float64) / ctx.num_blocks).contiguous()
        pm, pe = r.param_count()
        grad = torch.zeros(pm + pe, dtype=torch.float64, device=r.device)
        r.adjoint_passes(0, ctx.num_blocks * r.config.bands, ctx.first_pass, adj, grad)  # one launch
        gm = grad[:pm].view(mat.shape).to(ctx.mat_dtype)
        ge = grad[pm:].view(r.compiled.eem.shape).to(ctx.eem_dtype) if ctx.has_eem else None
        return gm, ge, None, None, None


def render_film(renderer, mat_f32, eem=None, first_pass=0, num_blocks=1):
    """Mean spectral film [B, H, W] (float64) of ``num_blocks`` blocks, differentiable in
    ``mat_f32`` [M, 6, B] and ``eem`` [E, B, B] (float32 or float64 tensors)."""
    return _RenderFilm.apply(mat_f32, eem, renderer, int(first_pass), int(num_blocks))


def film_to_xyz(film, cmf, scale):
    """XYZ [H, W, 3] of a [B, H, W] film: sum_b film[b] * cmf[b] * scale (color_rays, main.py:1617-1620)."""
    cmf = torch.as_tensor(cmf, dtype=film.dtype, device=film.device)
    return torch.einsum("bhw,bc->hwc", film, cmf) * scale


def material_table(renderer, dtype=torch.float32):
    """The uploaded material table [M, 6, B] as a tensor on the renderer's device."""
    return torch.as_tensor(renderer.compiled.mat_f32, dtype=dtype, device=renderer.device).clone()


def eem_table(renderer, dtype=torch.float32):
    """The uploaded EEM table [E, B, B] as a tensor on the renderer's device."""
    return torch.as_tensor(renderer.compiled.eem, dtype=dtype, device=renderer.device).clone()
