"""Device-resident gather instances and the seeded batched-gather workload.

A gather instance is what the reference's VPL integrator holds for one frame
(vpl.cc:496-520): a scene (aggregate on the device), one receiver per pixel from the
camera's primary hits, a VPL set traced from the lights, the clamp threshold
(0.1 x the mean unclamped contribution, the reference's "clamp at 0.1 x mean") and the
1 / num_emitted_photons scale.  Everything here stays on the device; the host only draws
sizes and keeps handles.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import rzk, scenegen as sg

MAX_BOUNCE = 3
TAU_PAIRS = 65536


@dataclasses.dataclass
class InstanceSpec:
    n_tris: int
    width: int
    height: int
    n_vpl: int
    seed: int

    @property
    def evals(self) -> int:
        return self.width * self.height * self.n_vpl


@dataclasses.dataclass
class GatherInstance:
    spec: InstanceSpec
    agg: "rzk.AggregateCuda"
    recv: object          # torch uint8 tensor of rzk_receiver records
    n_recv: int
    vpls: object          # torch uint8 tensor of rzk_vpl records
    n_vpl: int
    clamp_mode: int
    tau: float
    scale: float
    out: object           # torch float32 [n_recv, 3]

    def job(self):
        """The rzk_gather_job tuple of rzk.make_jobs."""
        return (self.agg, self.recv, self.n_recv, self.spec.width, self.vpls, self.n_vpl,
                self.clamp_mode, self.tau, self.scale, self.out)

    def gather(self, out=None, variant=0, n_chunks=0, stream=None):
        ev = rzk.VirtualPointLightCuda(self.agg, self.clamp_mode, self.tau)
        return ev.gather(self.recv, self.n_recv, self.vpls, self.n_vpl, scale=self.scale,
                         out=self.out if out is None else out, image_width=self.spec.width,
                         variant=variant, n_chunks=n_chunks, stream=stream)

    @property
    def device_bytes(self) -> int:
        return (self.agg.device_bytes + self.recv.numel() + self.vpls.numel()
                + self.out.numel() * 4)


def _log_uniform(rng, lo, hi):
    return math.exp(rng.uniform(math.log(lo), math.log(hi)))


def batch_specs(n: int = 64, seed: int = 2024, tris=(10_000, 500_000), side=(128, 1024),
                vpls=(1_000, 64_000)):
    """n instance sizes drawn log-uniform from `seed`: triangles, image side (a multiple
    of 8, square image) and VPL count."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        t = int(round(_log_uniform(rng, *tris)))
        s = int(round(_log_uniform(rng, *side) / 8.0)) * 8
        v = int(round(_log_uniform(rng, *vpls)))
        out.append(InstanceSpec(t, s, s, v, seed * 1000 + i))
    return out


def spawn_vpls(agg, seed: int, n_vpl: int, max_bounce: int = MAX_BOUNCE):
    """The first n_vpl VPLs in push order and the number of particles they came from."""
    particles = max(64, int(n_vpl * 0.8))
    gen = rzk.VplGeneratorCuda(agg)
    while True:
        vt, made = gen.spawn(seed, particles, max_bounce)
        if made >= n_vpl:
            break
        particles *= 2
    vt = vt[: n_vpl * 96].contiguous()
    last = rzk.records_from_device(vt[(n_vpl - 1) * 96:], sg.VPL_DTYPE)
    return vt, int(last["path"][0]) + 1


def make_instance(ctx, spec: InstanceSpec, clamp_mode: int = rzk.CLAMP_RADIANCE,
                  scene=None, agg=None) -> GatherInstance:
    """Builds the scene (unless `agg` is given), primary hits, VPLs and tau on the device."""
    import torch
    if agg is None:
        sc = scene if scene is not None else sg.room_filled(spec.n_tris, spec.width, spec.height, spec.seed)
        agg = rzk.AggregateCuda(ctx, sc)
        cam_spec = sc.camera
    else:
        cam_spec = dataclasses.replace(agg.scene.camera, width=spec.width, height=spec.height)
    cam = rzk.Camera(cam_spec)
    recv = agg.primary(cam)
    vt, emitted = spawn_vpls(agg, spec.seed, spec.n_vpl)
    ev = rzk.VirtualPointLightCuda(agg, clamp_mode, 1.0)
    tau = float(np.float32(0.1 * ev.mean_contribution(recv, cam.n_pixels, vt, spec.n_vpl, seed=spec.seed,
                                                      n_pairs=TAU_PAIRS)))
    out = torch.zeros((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    return GatherInstance(spec, agg, recv, cam.n_pixels, vt, spec.n_vpl, clamp_mode, tau,
                          1.0 / emitted, out)
