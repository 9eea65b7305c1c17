"""Scene builder (weave-sim_b200/csrc/scene.cpp): Kagome tracing, state layout, seeded inputs."""
import numpy as np
import pytest

import weavesim_b200 as ws


class Xoshiro:
    """xoshiro128** seeded by splitmix32, restated from web/js/rng.js:4-27 to check the builder's generator"""

    def __init__(self, seed):
        a = seed & 0xFFFFFFFF
        s = []
        for _ in range(4):
            a = (a + 0x9E3779B9) & 0xFFFFFFFF
            t = a ^ (a >> 16)
            t = (t * 0x21F0AAAD) & 0xFFFFFFFF
            t ^= t >> 15
            t = (t * 0x735A2D97) & 0xFFFFFFFF
            s.append(t ^ (t >> 15))
        self.s = s

    def u32(self):
        s = self.s
        rotl = lambda x, k: ((x << k) | (x >> (32 - k))) & 0xFFFFFFFF
        r = (rotl((s[1] * 5) & 0xFFFFFFFF, 7) * 9) & 0xFFFFFFFF
        t = (s[1] << 9) & 0xFFFFFFFF
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 11)
        return r

    def uniform(self):
        return ((self.u32() >> 5) * 67108864 + (self.u32() >> 6)) / 9007199254740992


def test_dome_small_counts():
    md = ws.configs.dome_small()
    # hexagon of side 4: 96 faces, 156 edges (24 on the boundary) = knots; 3 x 8 laths; 4 segments per knot spacing
    assert (md.n, md.m, md.p, md.K, md.n_strands) == (1176, 1152, 1128, 156, 24)
    assert len(md.anchor_node) == 48 and np.all(md.anchor_mask == 7)
    assert md.cross_enabled.sum() == 156 - 24           # boundary knots carry no contact without overhang
    assert abs(md.span - 7.5 * 0.35 * 2 / np.sqrt(3)) < 1e-9   # lath ends at the boundary edge midpoints


def test_shell_large_counts():
    md = ws.configs.shell_large()
    assert (md.K, md.n_strands) == (8190, 180)
    assert md.n == 81180 and md.m == 81000
    assert md.anchor_target is not None
    lift = md.anchor_target.reshape(-1, 3)[:, 2] - md.X.reshape(-1, 3)[md.anchor_node, 2]
    assert abs(lift.min()) < 1e-12 and abs(lift.max() - 2.0) < 1e-9


def test_strands_straight_and_alternating():
    md = ws.configs.dome_small(z_noise=0.0)
    X = md.X.reshape(-1, 3)
    off = md.node_offset
    h = 0.004
    for s in range(md.n_strands):
        P = X[off[s]:off[s + 1]]
        d = P[-1, :2] - P[0, :2]
        nrm = np.array([-d[1], d[0]]) / np.linalg.norm(d)
        assert np.abs((P[:, :2] - P[0, :2]) @ nrm).max() < 1e-9        # straight in plan on a regular lattice
        rows = np.arange(0, len(P), 4)                                  # knot rows (4 subdivisions)
        z = P[rows, 2]
        assert np.allclose(np.abs(z), h / 2) and np.all(z[1:] * z[:-1] < 0)   # over / under alternate


def test_crossing_sides_meet_in_plan():
    md = ws.configs.dome_small(z_noise=0.0)
    X = md.X.reshape(-1, 3)
    off = md.node_offset
    for c in range(md.K):
        pa = X[off[md.cross_strand[2 * c]] + int(md.cross_u[2 * c])]
        pb = X[off[md.cross_strand[2 * c + 1]] + int(md.cross_u[2 * c + 1])]
        assert np.linalg.norm(pa[:2] - pb[:2]) < 1e-9 and abs(abs(pa[2] - pb[2]) - 0.004) < 1e-9


def test_seeded_inputs_follow_the_reference_generator():
    md0 = ws.configs.dome_small(z_noise=0.0, seed=7)
    md1 = ws.configs.dome_small(z_noise=0.001, seed=7)
    dz = md1.X[2::3] - md0.X[2::3]
    # Box-Muller on xoshiro128** (rng.js:19-25), first pair
    r = Xoshiro(7)
    u = r.uniform()
    v = r.uniform()
    z0 = np.sqrt(-2 * np.log(u)) * np.cos(2 * np.pi * v)
    z1 = np.sqrt(-2 * np.log(u)) * np.sin(2 * np.pi * v)
    assert abs(dz[0] - 0.001 * z0) < 1e-15 and abs(dz[1] - 0.001 * z1) < 1e-15
    md2 = ws.configs.dome_stiff(seed=9)
    assert 0.1 <= md2.cross_mu.min() and md2.cross_mu.max() <= 0.5 and md2.cross_mu.std() > 0.05


def test_polyline_cases():
    import cases
    md = cases.crossing()
    assert (md.n, md.m, md.K) == (22, 20, 1)
    assert md.cross_u.tolist() == [5.0, 5.0]
    assert np.allclose(md.cross_nprev, [0, 0, 1])
    md = cases.cantilever(10)
    assert md.anchor_mask.tolist() == [63] and md.load_const[3 * md.tip + 2] == -10.0


def test_bad_scene_arguments():
    with pytest.raises(RuntimeError, match="positive"):
        ws.kagome(side=0, subdivisions=4, edge=0.4, width=0.04, height=0.004, E=1e10, G=6e8, density=500)


def test_shell_fixture_is_the_scene_builders_shell():
    """the CPU side of the benchmark reads the 20 m shell from oracle/scenes/shell_large.npz (so that process never loads
    the CUDA library); the fixture must be exactly what the scene builder makes"""
    import os
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "scenes", "shell_large.npz")
    a, b = ws.Model.load(path), ws.configs.shell_large()
    assert (a.n, a.m, a.p, a.K, a.n_strands, a.span) == (b.n, b.m, b.p, b.K, b.n_strands, b.span)
    assert a.params == b.params
    for k, v in b.__dict__.items():
        if isinstance(v, np.ndarray):
            w = getattr(a, k)
            assert w.dtype == v.dtype and np.array_equal(w, v), k
