"""The committed model tables are the generator's output, and the generator
reproduces the reference's own header (CPU only).

tests/golden/ref_model_tables.npz (tests/golden/make_model_tables.py) holds
the reference header's numbers (src/g1_model.h:15-359, parsed as text) and
the output of g1sim_b200/model/gen_model.py run on the reference's MJCF.
Both the C header that the device code compiles (csrc/g1_model_data.h) and
its Python twin (model/g1_model_data.py) must equal the generator's output
bit for bit -- a hand edit of either fails here -- and the generator's
output must equal the reference header (derived values -- the rotated
inertias and the damping gains from the mass-matrix diagonal -- to a few
ulps, since MuJoCo and the generator round differently)."""
import os
import re

import numpy as np
import pytest

from g1sim_b200.model import g1_model_data as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLES = ("parent", "tree_pos", "tree_quat", "mass", "com", "inertia_com", "jnt_axis", "jnt_anchor", "armature",
          "damping", "jnt_range", "act_kp", "act_kv", "act_frclim", "contact_body", "contact_pos", "qpos_stand")
DERIVED = ("inertia_com", "act_kv")


@pytest.fixture(scope="module")
def fixture():
    return np.load(os.path.join(ROOT, "tests", "golden", "ref_model_tables.npz"))


def flat(v):
    a = []
    for r in v:
        a.extend(r if isinstance(r, (list, tuple)) else [r])
    return np.array(a, dtype=np.float64)


def header_tables():
    text = open(os.path.join(ROOT, "g1sim_b200", "csrc", "g1_model_data.h")).read()
    out = {}
    for name in TABLES:
        m = re.search(r"\bg1m_%s\[(\d+)\]\s*=\s*\{([^}]*)\}" % name, text)
        assert m, name
        vals = np.array([float(x) for x in m.group(2).replace("\n", " ").split(",") if x.strip()])
        assert vals.size == int(m.group(1))
        out[name] = vals
    return out


@pytest.mark.parametrize("name", TABLES)
def test_committed_tables_are_the_generator_output(fixture, name):
    gen = fixture[f"gen_{name}"]
    assert np.array_equal(flat(getattr(M, name)), gen), name
    assert np.array_equal(header_tables()[name], gen), name


@pytest.mark.parametrize("name", TABLES)
def test_generator_reproduces_reference_header(fixture, name):
    gen, ref = fixture[f"gen_{name}"], fixture[f"ref_{name}"]
    assert gen.shape == ref.shape
    if name in DERIVED:
        err = np.abs(gen - ref) / np.maximum(np.abs(ref), 1e-12)
        assert err.max() < 1e-14, (name, err.max())
    else:
        assert np.array_equal(gen, ref), name
