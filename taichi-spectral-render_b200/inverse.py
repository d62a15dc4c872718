"""Inverse rendering of spectral material parameters (the differentiable workload).

The box scene with the HG medium and the fluorescent back wall, with 79
unknowns: the per-band albedos of the left and right walls (2 x 25), the
medium's per-band absorption sigma_a (25), its HG anisotropy g, and the GGX
roughnesses of the fluorescent back wall and the left and right walls (3):
under the reference's surface model (main.py:1384-1412) a wall of roughness
above 0.008 carries a GGX lobe with the Fresnel term of its n = 1.5 coating
over an Oren-Nayar diffuse term of sigma = roughness * pi / 2, so each
roughness moves both.
The medium's boundary stays a smooth dielectric: under the reference's
estimator a rough dielectric boundary transmits nothing (its Smith term
clamps the refracted cosine to zero), which would hide the medium.  A target image is
rendered from hidden parameters, and Adam fits the parameters from an
initial guess by minimising the L2 distance of the XYZ images, each step a
forward render and a path-replay adjoint of the same paths
(autodiff.render_film).

Parameters live in an unconstrained space (albedo = sigmoid, sigma_a = exp,
g = 0.95 tanh, roughness = sigmoid) and are mapped onto the material table
[M][6][B] with torch operations, so autograd composes the mapping with the
adjoint's table gradient.
"""
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import autodiff
from .configs import volume_scene

BACK, LEFT, RIGHT, MEDIUM = 3, 5, 6, 8  # material ids of volume_scene (walls 1..6, light 7, medium 8)


@dataclass
class Params:
    albedo_left: torch.Tensor   # [B] in (0, 1)
    albedo_right: torch.Tensor  # [B]
    sigma_a: torch.Tensor       # [B] 1/m
    g: torch.Tensor             # scalar in (-0.95, 0.95)
    roughness: torch.Tensor     # [3]: back, left, right wall

    @staticmethod
    def from_scene_params(p, device):
        f = lambda x: torch.as_tensor(np.asarray(x, np.float64), device=device)
        return Params(f(p["albedo_left"]), f(p["albedo_right"]), f(p["sigma_a"]), f(p["g"]), f(p["roughness"]))

    def count(self):
        return sum(int(np.prod(t.shape)) if t.dim() else 1 for t in (self.albedo_left, self.albedo_right,
                                                                      self.sigma_a, self.g, self.roughness))


def to_unconstrained(p):
    logit = lambda x: torch.log(x.clamp(1e-4, 1 - 1e-4)) - torch.log1p(-x.clamp(1e-4, 1 - 1e-4))
    return [logit(p.albedo_left), logit(p.albedo_right), torch.log(p.sigma_a.clamp_min(1e-6)),
            torch.atanh((p.g / 0.95).clamp(-0.999, 0.999)), logit(p.roughness)]


def from_unconstrained(u):
    return Params(torch.sigmoid(u[0]), torch.sigmoid(u[1]), torch.exp(u[2]), 0.95 * torch.tanh(u[3]),
                  torch.sigmoid(u[4]))


def material_table(base, p, wavelengths_nm):
    """The material table [M][6][B] with the parameters written in (differentiable)."""
    lam = torch.as_tensor(np.asarray(wavelengths_nm, np.float64) * 1e-9, device=base.device)
    mat = base.to(torch.float64).clone()
    k_of_albedo = lambda rho: lam * (1.0 / rho - 1.0) / (4.0 * math.pi)  # sigma_s = 1 gives albedo rho
    mat[LEFT, 1] = k_of_albedo(p.albedo_left)
    mat[RIGHT, 1] = k_of_albedo(p.albedo_right)
    mat[MEDIUM, 1] = p.sigma_a * lam / (4.0 * math.pi)
    mat[MEDIUM, 5] = p.g * torch.ones_like(lam)
    mat[BACK, 2] = p.roughness[0] * torch.ones_like(lam)
    mat[LEFT, 2] = p.roughness[1] * torch.ones_like(lam)
    mat[RIGHT, 2] = p.roughness[2] * torch.ones_like(lam)
    return mat


def scene_params(seed):
    """79 parameters drawn from ``seed``: the wall albedos and sigma_a(lambda) as the
    scene generator draws them for that seed (logistic reflectances, sums of two
    Gaussians), g uniform in [0.3, 0.9] and roughnesses uniform in [0.05, 0.5]."""
    _, _, ex = volume_scene(seed=seed, width=8, height=8, medium_slices=8, medium_stacks=9)
    p = dict(ex["params"])
    rng = np.random.default_rng(seed + 10_000)
    p["g"] = float(rng.uniform(0.3, 0.9))
    p["roughness"] = rng.uniform(0.05, 0.5, size=3).tolist()
    return p


def run(renderer, target_xyz, init, iterations=200, lr=1e-2, blocks=2, first_pass=1 << 20, log=None):
    """Adam on the unconstrained parameters; returns the fitted Params and the loss history.

    Each iteration renders ``blocks`` spectral blocks (new random streams per
    iteration) and back-propagates through the same paths."""
    r = renderer
    base = autodiff.material_table(r)
    eem = autodiff.eem_table(r)
    lam = r.config.wavelengths()
    u = [t.detach().clone().requires_grad_(True) for t in to_unconstrained(init)]
    opt = torch.optim.Adam(u, lr=lr)
    hist = []
    B = r.config.bands
    for it in range(iterations):
        opt.zero_grad()
        p = from_unconstrained(u)
        mat = material_table(base, p, lam)
        film = autodiff.render_film(r, mat, eem, first_pass=first_pass + it * blocks * B, num_blocks=blocks)
        xyz = autodiff.film_to_xyz(film, r.compiled.cmf, r.cmf_scale)
        loss = ((xyz - target_xyz) ** 2).mean()
        loss.backward()
        opt.step()
        hist.append(float(loss.detach()))
        if log is not None:
            log(it, hist[-1], p)
    return from_unconstrained([t.detach() for t in u]), hist


def render_target(renderer, params, blocks):
    """XYZ image of ``params`` at ``blocks`` spectral blocks (no gradient)."""
    r = renderer
    base = autodiff.material_table(r)
    mat = material_table(base, params, r.config.wavelengths()).float()
    with torch.no_grad():
        film = autodiff.render_film(r, mat, autodiff.eem_table(r), first_pass=0, num_blocks=blocks)
        return autodiff.film_to_xyz(film, r.compiled.cmf, r.cmf_scale)


def image_loss(renderer, params, target_xyz, blocks=2, first_pass=1 << 20):
    """The loss of ``run`` at fixed parameters (e.g. the hidden ones: the noise floor)."""
    r = renderer
    mat = material_table(autodiff.material_table(r), params, r.config.wavelengths()).float()
    with torch.no_grad():
        film = autodiff.render_film(r, mat, autodiff.eem_table(r), first_pass=first_pass, num_blocks=blocks)
        xyz = autodiff.film_to_xyz(film, r.compiled.cmf, r.cmf_scale)
        return float(((xyz - target_xyz) ** 2).mean())


def parameter_error(p, q):
    """Relative L2 error of each parameter group of p against q."""
    out = {}
    for name in ("albedo_left", "albedo_right", "sigma_a", "g", "roughness"):
        a, b = getattr(p, name), getattr(q, name)
        out[name] = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b).clamp_min(1e-12))
    return out


NAMES = ("albedo_left", "albedo_right", "sigma_a", "g", "roughness")


def gradient_check(renderer, params, h=1e-3, blocks=40, first_pass=1 << 22, seed=0, groups=10):
    """The adjoint against central finite differences, parameter by parameter.

    The functional is L(theta) = sum(w * film(theta)) with a fixed random
    weight w per film cell (the adjoint of any image loss is such a weighted
    film).  Adjoint side: autodiff.render_film over ``blocks`` spectral blocks
    and backward through the parameter mapping of ``material_table``.
    Finite-difference side: L(theta + h e_i) and L(theta - h e_i) rendered on
    the same passes (common random numbers), with the step h relative to each
    of the 79 physical parameters (albedos, sigma_a [1/m], g, roughnesses:
    step h * |value|, so that no step leaves a parameter's domain -- sigma_a
    spans orders of magnitude over the bands); the per-block differences give
    the standard error of the estimate.  The adjoint is itself a Monte Carlo
    estimate (its score terms add variance of their own): it is computed over
    ``groups`` equal runs of consecutive blocks, whose spread gives its
    standard error, and its mean is the gradient over all ``blocks``.
    Returns a list of dicts (name, index, value, step, adjoint, adjoint_sem,
    fd, fd_sem)."""
    r = renderer
    B = r.config.bands
    base = autodiff.material_table(r)
    eem = autodiff.eem_table(r)
    lam = r.config.wavelengths()
    gen = torch.Generator(device=r.device)
    gen.manual_seed(seed)
    w = torch.rand((B, r.config.height, r.config.width), dtype=torch.float64, device=r.device, generator=gen)
    if groups < 1 or blocks % groups:
        groups = 1
    per = blocks // groups
    grads = {n: [] for n in NAMES}
    for g in range(groups):
        leaves = {n: getattr(params, n).detach().clone().to(torch.float64).requires_grad_(True) for n in NAMES}
        film = autodiff.render_film(r, material_table(base, Params(**leaves), lam), eem,
                                    first_pass=first_pass + g * per * B, num_blocks=per)
        (film * w).sum().backward()
        for n in NAMES:
            grads[n].append(leaves[n].grad.detach().reshape(-1))
    r.record_paths(0, 0)
    gstack = {n: torch.stack(grads[n]) for n in NAMES}  # [groups, count]

    def per_block(p):
        r.update_materials(material_table(base, p, lam).float().contiguous(), None)
        r.clear_pixel_space()
        out = np.zeros(blocks)
        for b in range(blocks):
            r.cast_rays_bundle(0, B, pass_idx=first_pass + b * B)
            out[b] = float((r.block_film * w).sum())
            r.average_and_reset_block(b + 1)  # clears the block film for the next one
        return out

    rows = []
    for name in NAMES:
        val = getattr(params, name).detach().to(torch.float64)
        flat = val.reshape(-1)
        grad = gstack[name].mean(0)
        grad_sem = (gstack[name].std(0, unbiased=True) / groups ** 0.5 if groups > 1
                    else torch.full_like(grad, float("nan")))
        for i in range(flat.numel()):
            lo = {n: getattr(params, n).detach().to(torch.float64) for n in NAMES}
            hi = dict(lo)
            step = h * max(abs(float(flat[i])), 1e-12)
            dp = torch.zeros_like(flat)
            dp[i] = step
            hi[name] = (flat + dp).reshape(val.shape)
            lo[name] = (flat - dp).reshape(val.shape)
            d = (per_block(Params(**hi)) - per_block(Params(**lo))) / (2.0 * step)
            rows.append({"name": name, "index": i, "value": float(flat[i]), "step": step, "adjoint": float(grad[i]),
                         "adjoint_sem": float(grad_sem[i]), "fd": float(d.mean()),
                         "fd_sem": float(d.std(ddof=1) / np.sqrt(blocks))})
    # leave the renderer with the unperturbed tables
    r.update_materials(material_table(base, params, lam).float().contiguous(), None)
    return rows

