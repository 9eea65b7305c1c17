"""The gridshell workloads of this solver, built with the scene builder (SI units: m, N, Pa).

* ``dome_small``   — 3 m hexagonal plan, 3 lath families at 0/60/120°, 8 laths per family at 0.35 m, 5 cm segments,
                     40×4 mm timber laths (E 10 GPa, G 0.6 GPa, 500 kg/m³), μ 0.3, perimeter lath ends pinned and
                     moved 0.25 m radially inward, flat start with N(0, 1 mm) z-noise, self-weight on.
* ``shell_large``  — the same lath model on a 20 m plan: 60 laths per family at 0.33 m, 4 cm segments (5 per knot
                     spacing), support ends lifted 0–2 m by a smooth seeded field, μ 0.3.
* ``dome_stiff``   — ``dome_small`` with 25×3 mm laths, E 12 GPa, per-crossing μ ~ U(0.1, 0.5).
* ``batch_mixed``  — independent gridshells drawn from a seed: laths per family U{6..40}, span U(2, 12) m, thickness
                     U(3, 6) mm, width U(30, 60) mm, E U(8, 14) GPa, μ U(0.1, 0.5), inward displacement U(3 %, 10 %)
                     of the span, ~5 cm segments.  The inward displacement is read as the reduction of the span: the
                     supports on opposite sides each move radially by half of it, so every support moves by
                     U(1.5 %, 5 %) of the span.

Contact penalties (strength = stick_strength = 1e5 N/m) follow the reference's thin-lath example scene
(examples/scenes/dualv5dome_cm.json: 40 mm laths, 1000 N/cm); its default 1e4 N/mm belongs to 60×30 mm sections.
The supports move to their targets over ``disp_ramp_iter`` iterations after the warm-up.

Lattice sizing: laths per family = 2·side of the hexagon; family spacing s = a·√3/2 for triangle edge a; knot spacing
along a lath = a/2; subdivisions = round((a/2) / segment length).
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import default_params, kagome

SQ3 = math.sqrt(3.0)


def _sub(edge, seg):
    return max(1, int(round(0.5 * edge / seg)))


def dome_small(seed=1, **over):
    edge = 0.35 * 2 / SQ3
    kw = dict(side=4, subdivisions=_sub(edge, 0.05), edge=edge, width=0.040, height=0.004, E=10e9, G=0.6e9,
              density=500.0, mu=0.3, inward=0.25, z_noise=0.001, gravity=True, seed=seed)
    kw.update(over)
    kw.setdefault("params", default_params(disp_ramp_iter=3000, max_iter=50000, strength=1e5, stick_strength=1e5))
    return kagome(**kw)


def shell_large(seed=2, **over):
    edge = 0.33 * 2 / SQ3
    kw = dict(side=30, subdivisions=_sub(edge, 0.04), edge=edge, width=0.040, height=0.004, E=10e9, G=0.6e9,
              density=500.0, mu=0.3, lift=2.0, z_noise=0.0, gravity=True, seed=seed)
    kw.update(over)
    kw.setdefault("params", default_params(disp_ramp_iter=5000, max_iter=100000, strength=1e5,
                                                 stick_strength=1e5))
    return kagome(**kw)


def dome_stiff(seed=3, **over):
    kw = dict(width=0.025, height=0.003, E=12e9, mu_range=(0.1, 0.5), seed=seed)
    kw.update(over)
    return dome_small(**kw)


def batch_draw(rng: np.random.Generator):
    """One gridshell of the mixed batch: keyword arguments of ``kagome``."""
    laths = int(rng.integers(6, 41))
    side = max(3, laths // 2)
    span = float(rng.uniform(2.0, 12.0))
    edge = span / (2 * side)
    t = float(rng.uniform(0.003, 0.006))
    w = float(rng.uniform(0.030, 0.060))
    E = float(rng.uniform(8e9, 14e9))
    mu = float(rng.uniform(0.1, 0.5))
    inward = float(rng.uniform(0.03, 0.10)) * span * 0.5     # radial move of each support: half the span reduction
    return dict(side=side, subdivisions=_sub(edge, 0.05), edge=edge, width=w, height=t, E=E, G=0.06 * E,
                density=500.0, mu=mu, inward=inward, z_noise=0.001, gravity=True,
                seed=int(rng.integers(1, 2 ** 31)), params=default_params(disp_ramp_iter=3000, max_iter=50000, strength=1e5, stick_strength=1e5))


def batch_mixed(count=512, seed=4, max_nodes=None):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        kw = batch_draw(rng)
        md = kagome(**kw)
        if max_nodes and md.n > max_nodes:
            continue
        out.append(md)
    return out
