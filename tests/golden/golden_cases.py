"""Small cases shared by the golden-fixture generator and the tests that read the fixtures.

Each case is built from ``celeris_b200.cases.small_case`` (deterministic, seeded) plus the
variations named here; ``STEPS`` physical steps are taken before the state is recorded.
"""
from __future__ import annotations

import numpy as np

from celeris_b200 import cases

STEPS = 20
NAMES = ["solid", "mixed", "sponge", "irregular", "uts", "solid_wide", "irregular_sea_level", "adaptive_manning",
         "nlsw", "adaptive_ab3"]


def golden_case(name: str):
    """Returns (params, z, bnx, bny, keep): keep holds buffers the params point into."""
    keep = []
    if name in ("solid", "mixed", "sponge", "irregular", "uts"):
        p, z, bnx, bny = cases.small_case(40, 24, name, correction_steps=1)
    elif name == "solid_wide":
        p, z, bnx, bny = cases.small_case(40, 24, "solid", correction_steps=1)
        p.west.width, p.east.width, p.south.width, p.north.width = 3, 4, 5, 3
    elif name == "irregular_sea_level":
        p, z, bnx, bny = cases.small_case(40, 24, "irregular", correction_steps=1)
        p.west.sea_level, p.south.sea_level = 0.05, 0.02
    elif name == "nlsw":
        # model type NLSW: identity tridiagonal systems, dispersion terms kept (engine.cpp:2625, 4127);
        # those terms are then explicit, so the grid is 4 m (depth / dx ~ 1) with the Courant number kept
        p, z, bnx, bny = cases.small_case(40, 24, "mixed", correction_steps=1)
        p.boussinesq = 0
        p.width, p.length, p.timestep = 4 * p.width, 4 * p.length, 4 * p.timestep
    elif name == "adaptive_ab3":
        # adaptive predictor every step (no corrector): the variable-step AB3 of compute.hlsl:766-780
        p, z, bnx, bny = cases.small_case(44, 26, "mixed", correction_steps=0)
        p.adaptive = 1
        p.timestep *= 0.5
    elif name == "adaptive_manning":
        p, z, bnx, bny = cases.small_case(37, 29, "sponge", correction_steps=2)
        p.adaptive = 1
        p.manning, p.friction, p.dissipation_threshold = 1, 0.03, 0.2
    else:
        raise KeyError(name)
    if name == "uts":
        keep += cases.attach_uts(p, "west", np.array(
            [[0, 0, 0, 0], [5, 0.2, 0.1, 0], [10, -0.1, 0.05, 0.02], [100, 0, 0, 0]], float))
        keep += cases.attach_uts(p, "north", np.array([[0, 0, 0, 0], [3, 0.05, 0, 0.01], [100, 0.1, 0, 0]], float))
    return p, z, bnx, bny, keep


def bottom_case():
    """A seeded .cbf grid coarser than the mesh, so the bilinear sampling is exercised."""
    rng = np.random.default_rng(4242)
    bnx, bny = 23, 17
    z = (-4.0 + 0.2 * np.arange(bnx)[None, :] + 0.3 * rng.standard_normal((bny, bnx))).astype(np.float32)
    return dict(nx=40, ny=24, width=39.0, length=23.0, swl=0.0, gravity=9.81, bnx=bnx, bny=bny, z=z)


def write_cbf(path: str, z: np.ndarray) -> None:
    """The reference's .cbf layout: [nx]/[ny] header lines, a '=' line, then ny rows of nx values."""
    bny, bnx = z.shape
    with open(path, "w") as f:
        f.write(f"[nx] {bnx}\n[ny] {bny}\n====================================\n")
        for row in z:
            f.write(" ".join(f"{float(v):.9g}" for v in row) + "\n")
