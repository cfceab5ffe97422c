"""Differentiable rendering through the path-replay adjoint (rs_backward).

`render_sequence(params, renderer, cameras)` renders a camera sequence with the ReservoirSplatting
pass and is differentiable with respect to `params`, a (materials x 8) float32 tensor in the order
baseColor.xyz, roughness, emissive.xyz, metallic (the layout of the first eight floats of a material
record).  Forward keeps one checkpoint per frame (the final reservoirs, 144 bytes per pixel); backward
calls rs_backward once per frame with that frame's checkpoint and d loss / d image.  Every column is
differentiated; for a spec-gloss material the baseColor columns are its diffuse colour, the roughness
column its glossiness, and its metallic column (derived from its colours) gets no gradient.

The estimator and its conditions (emissive triangles and an environment map, no analytic lights;
the TinyUniform generator for paths of four or more vertices) are those of rs_backward.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ReservoirSplatting

PARAM_WIDTH = 8  # baseColor.xyz, roughness, emissive.xyz, metallic


class Renderer:
    """A pass configured for differentiation plus the scene's full material records."""

    def __init__(self, scene, props: dict | None = None, width: int = 512, height: int = 512):
        props = dict(props or {})
        props.setdefault("maxSurfaceBounces", 1)
        self.pass_ = ReservoirSplatting(props, width, height)
        self.pass_.set_scene(scene)
        self.materials = np.array(scene.materials, np.float32).reshape(len(scene.materials), -1).copy()
        self.width, self.height = width, height

    @property
    def num_materials(self) -> int:
        return len(self.materials)

    def params(self) -> torch.Tensor:
        return torch.from_numpy(self.materials[:, :PARAM_WIDTH].copy())

    def apply(self, params: torch.Tensor):
        self.materials[:, :PARAM_WIDTH] = params.detach().to("cpu", torch.float32).numpy()
        self.pass_.set_materials(self.materials)

    def render(self, cameras, keep_checkpoints: bool = True):
        """Renders the sequence from a fresh temporal history; returns (images, checkpoints)."""
        stream = torch.cuda.current_stream().cuda_stream
        images = torch.empty((len(cameras), self.height, self.width, 4), dtype=torch.float32, device="cuda")
        ckpts = []
        nbytes = self.pass_.checkpoint_bytes()
        self.pass_.reset()
        for f, cam in enumerate(cameras):
            self.pass_.execute(cam, color_ptr=images[f].data_ptr(), stream=stream, should_reset=(f == 0))
            if keep_checkpoints:
                ck = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
                self.pass_.checkpoint(ck.data_ptr(), stream)
                ckpts.append(ck)
        return images, ckpts

    def backward(self, grad_images: torch.Tensor, ckpts) -> torch.Tensor:
        stream = torch.cuda.current_stream().cuda_stream
        grad = torch.zeros((self.num_materials, PARAM_WIDTH), dtype=torch.float32, device="cuda")
        g = grad_images.to(device="cuda", dtype=torch.float32).contiguous()
        for f, ck in enumerate(ckpts):
            self.pass_.backward(g[f].data_ptr(), grad.data_ptr(), ck.data_ptr(), stream)
        return grad


class _RenderSequence(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, renderer, cameras):
        renderer.apply(params)
        images, ckpts = renderer.render(cameras)
        ctx.renderer = renderer
        ctx.ckpts = ckpts
        ctx.param_device = params.device
        return images

    @staticmethod
    def backward(ctx, grad_images):
        grad = ctx.renderer.backward(grad_images, ctx.ckpts)
        ctx.ckpts = None
        return grad.to(ctx.param_device), None, None


def render_sequence(params: torch.Tensor, renderer: Renderer, cameras) -> torch.Tensor:
    """Images (frames x H x W x 4, CUDA) of `cameras`, differentiable with respect to `params`."""
    return _RenderSequence.apply(params, renderer, list(cameras))
