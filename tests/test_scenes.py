"""Seeded scene builders: sizes match the workload definitions and builds are deterministic."""
import numpy as np

from natsel_b200 import scenes
from oracle import pyoracle


class Recorder:
    """Records the construction calls a builder makes."""

    def __init__(self):
        self.calls = []
        self.body_types = []

    def create_body(self, type=2, position=(0, 0, 0), rotation=(0, 0, 0, 1), **kw):
        self.body_types.append(type)
        self.calls.append(("body", type, tuple(position), tuple(rotation), tuple(sorted(kw.items()))))
        return len(self.body_types) - 1

    def create_box(self, b, hx, hy, hz, **kw):
        self.calls.append(("box", b, hx, hy, hz, tuple(sorted(kw.items()))))

    def create_sphere(self, b, r, center=(0, 0, 0), **kw):
        self.calls.append(("sphere", b, r, tuple(sorted(kw.items()))))

    def create_capsule(self, b, c1, c2, r, **kw):
        self.calls.append(("capsule", b, tuple(c1), tuple(c2), r, tuple(sorted(kw.items()))))

    def create_revolute(self, a, b, fa, fb, **kw):
        self.calls.append(("revolute", a, b, tuple(fa), tuple(fb), tuple(sorted(kw.items()))))


def test_box_pyramid_shape():
    r = Recorder()
    info = scenes.box_pyramid(r)
    assert info["dynamic_bodies"] == 210
    assert sum(1 for c in r.calls if c[0] == "box") == 211
    assert r.body_types.count(2) == 210


def test_large_pile_mix():
    r = Recorder()
    info = scenes.large_pile(r)
    assert info["dynamic_bodies"] == 10000
    kinds = [c[0] for c in r.calls if c[0] in ("box", "sphere", "capsule")]
    assert kinds.count("box") == 6001 and kinds.count("sphere") == 2500 and kinds.count("capsule") == 1500
    ys = [c[2][1] for c in r.calls if c[0] == "body" and c[1] == 2]
    assert 1.0 <= min(ys) and max(ys) <= 61.0


def test_jointed_chains_counts():
    r = Recorder()
    info = scenes.jointed_chains(r)
    assert info["dynamic_bodies"] == 2000 * 24 + 4000
    assert info["joints"] == 48000


def test_builders_are_deterministic():
    for name in ("box_pyramid", "large_pile", "jointed_chains"):
        a, b = Recorder(), Recorder()
        kw = {"n": 500} if name == "large_pile" else ({"chains": 20, "boxes": 40} if name == "jointed_chains" else {})
        scenes.BUILDERS[name](a, **kw)
        scenes.BUILDERS[name](b, **kw)
        assert a.calls == b.calls


def test_cos_sin_matches_reference_identities():
    c, s = scenes.compute_cos_sin(0.0)
    assert c == np.float32(1.0) and s == np.float32(0.0)
    for x in np.linspace(-7.0, 7.0, 57):
        c, s = scenes.compute_cos_sin(x)
        assert abs(float(c) - np.cos(x)) < 2e-3 and abs(float(s) - np.sin(x)) < 2e-3


def test_oracle_scene_hash_is_reproducible():
    hs = []
    for _ in range(2):
        w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS["box_pyramid"])
        scenes.box_pyramid(w)
        w.step(1.0 / 60.0, 4)
        hs.append(w.state_hash())
    assert hs[0] == hs[1]
