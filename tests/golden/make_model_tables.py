#!/usr/bin/env python3
"""Generate tests/golden/ref_model_tables.npz from the REFERENCE's files.

Two sets of model tables, both taken where the reference sources lie (the
development container only):
  ref_<name>  the numbers of the reference's checked-in header
              (src/g1_model.h:15-359, written by its MuJoCo-based
              model/gen_model.py), parsed as text;
  gen_<name>  this repository's generator (g1sim_b200/model/gen_model.py,
              no MuJoCo) run on the reference's MJCF (model/g1_stripped.xml,
              model/g1_raw.xml).
tests/test_model_tables.py checks that the committed tables are exactly the
generator's output and that the generator reproduces the reference header.

Run:  python tests/golden/make_model_tables.py [<reference root>]
      (default: $REF_SRC, else /root/reference)
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from g1sim_b200.model import gen_model  # noqa: E402

TABLES = ("parent", "tree_pos", "tree_quat", "mass", "com", "inertia_com", "jnt_axis", "jnt_anchor", "armature",
          "damping", "jnt_range", "act_kp", "act_kv", "act_frclim", "contact_body", "contact_pos", "qpos_stand")


def parse_header(path):
    text = open(path).read()
    out = {}
    for name in TABLES:
        m = re.search(r"\bg1_%s\[(\d+)\]\s*=\s*\{([^}]*)\}" % name, text)
        assert m, name
        body = re.sub(r"\bR\(([^)]*)\)", r"\1", m.group(2))  # the header wraps reals as R(x)
        vals = [float(x) for x in body.replace("\n", " ").split(",") if x.strip()]
        assert len(vals) == int(m.group(1)), (name, len(vals))
        out[name] = np.array(vals)
    return out


def flat(v):
    a = []
    for r in v:
        a.extend(r if isinstance(r, (list, tuple)) else [r])
    return np.array(a, dtype=np.float64)


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_SRC", "/root/reference")
    hdr = parse_header(os.path.join(ref, "src", "g1_model.h"))
    data = gen_model.build(os.path.join(ref, "model"))
    out = {f"ref_{k}": v for k, v in hdr.items()}
    out.update({f"gen_{k}": flat(data[k]) for k in TABLES})
    np.savez_compressed(os.path.join(HERE, "ref_model_tables.npz"), **out)
    for k in TABLES:
        a, b = out[f"gen_{k}"], out[f"ref_{k}"]
        print(f"{k:14s} max rel diff gen vs ref {float((np.abs(a - b) / np.maximum(np.abs(b), 1e-300)).max()):.2e}")


if __name__ == "__main__":
    main()
