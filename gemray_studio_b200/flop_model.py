"""Algorithmic FLOP model of one path-sample, from the instrumented kernel's event
tallies (gr_event_counts).

Counting rule: add / sub / mul / div / sqrt = 1 flop, fused multiply-add = 2;
compares, min / max / abs / floor / selects = 0; each transcendental (sin, cos, atan,
atan2, acos, libm exp) is one SFU op counted separately, not as flops.  The
reference's polynomial exp (simd/exp_poly.rs) is ordinary arithmetic: 22 flops.

Per-event costs are static counts of the arithmetic in gemray_studio_b200/csrc
(gr_device.cuh, gr_trace.cuh), which follows the reference's operation order
op for op (crates/gemray/src/optics/raytracer/*.rs).
"""
from __future__ import annotations

from dataclasses import dataclass

# per plane of every intersection test (intersect.rs:93-132 / slab.rs:140-152):
# denom 3 mul + 2 add, side 3 mul + 3 add, t 1 div
PLANE = 12
INIT = 258             # sampler (48) + camera ray (34) + per-channel lambda/dispersion (8 x 22)
INIT_BAND = 6          # per absorption band per channel per set (Gaussian band sum)
HIT = 54               # hit point, plane-of-incidence normal, incidence geometry, n1/n2, origin update
ROTATION = 264         # frame-rotation Mueller product over 8 channels (+3 SFU)
ABSORB = 1508          # pleochroic Beer-Lambert over 8 channels (+24 SFU)
ANISO = 85             # uniaxial n_eff(theta) for 8 channels (+3 SFU)
CH_SPLIT = 3           # per channel of a reflect/TIR/refract event: n1/n2, sin^2 t
CH_TIR = 42            # channel past its critical angle: TIR phase + retarder (+3 SFU)
CH_FRESNEL = 58        # channel partial reflection: r_s, r_p, Mueller, path pdf
TIR = 12               # reflected wave normal
PARTIAL = 19           # hero r_s / r_p / r_unpol and the branch draw
REFLECT = 13           # 1/r_unpol and the reflected wave normal
REFRACT = 28           # hero refracted wave normal
CH_REFRACT = 106       # per transmitting channel: direction, t_s/t_p, Mueller, pdf
WALKOFF = 58           # extraordinary Poynting direction (+5 SFU)
ROULETTE = 34
FINISH = 1707          # spectral MIS + 8-channel CMF (7 polynomial lobes each) + von Kries
ESCAPE = {0: 208, 1: 1090, 2: 263}  # uniform / studio / lat-long environment, 8 channels

SFU = {"rotation": 3, "absorb": 24, "aniso": 3, "ch_tir": 3, "walkoff": 5}
SFU_ESCAPE = {0: 24, 1: 8, 2: 26}


@dataclass
class Model:
    flops: float
    sfu: float
    paths: int

    @property
    def flops_per_sample(self) -> float:
        return self.flops / max(1, self.paths)


def evaluate(counts: dict[str, int], n_planes: int, env_mode: int, n_bands: int = 0) -> Model:
    c = counts
    reflect_type = c["tir"] + c["reflect"]
    ch_fresnel = 8 * reflect_type - c["channel_tir"]
    flops = (
        c["paths"] * (INIT + 16 * n_bands * INIT_BAND + FINISH)
        + c["bounces"] * PLANE * n_planes
        + (c["bounces"] - c["escapes"]) * HIT
        + c["rotations"] * ROTATION
        + c["absorb"] * ABSORB
        + c["aniso_bounces"] * ANISO
        + 8 * (reflect_type + c["refract"]) * CH_SPLIT
        + c["channel_tir"] * CH_TIR
        + max(0, ch_fresnel) * CH_FRESNEL
        + c["tir"] * TIR
        + (c["reflect"] + c["refract"]) * PARTIAL
        + c["reflect"] * REFLECT
        + c["refract"] * REFRACT
        + c["channel_refract"] * CH_REFRACT
        + c["walkoff"] * WALKOFF
        + c["roulette"] * ROULETTE
        + c["escapes"] * ESCAPE[env_mode]
    )
    sfu = (
        c["rotations"] * SFU["rotation"] + c["absorb"] * SFU["absorb"] + c["aniso_bounces"] * SFU["aniso"]
        + c["channel_tir"] * SFU["ch_tir"] + c["walkoff"] * SFU["walkoff"] + c["escapes"] * SFU_ESCAPE[env_mode]
        + c["paths"] * 16 * n_bands
    )
    return Model(flops=float(flops), sfu=float(sfu), paths=int(c["paths"]))
