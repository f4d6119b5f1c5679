#!/usr/bin/env python3
"""Build the G1 model tables from the MJCF files, without MuJoCo.

The reference compiles the Menagerie MJCF with MuJoCo and bakes the compiled
values into a C header (reference: model/gen_model.py:80-187, output
src/g1_model.h).  MuJoCo is not installable here, so this script restates the
few compiler steps that the G1 needs in plain numpy:

* body tree in document order, parent indices        (gen_model.py:99-100)
* body pos / unit quaternion (MuJoCo normalises)      (gen_model.py:101-102)
* inertia about the COM in the body frame, R diag R^T (gen_model.py:105-109)
* hinge axis / anchor / armature / damping / range    (gen_model.py:111-120)
* position-servo kp, kv from ``dampratio`` and force limits (gen_model.py:125-135)
  kv = 2 * dampratio * sqrt(kp * M0[j]) where M0 is the joint-space mass
  matrix diagonal at qpos0 (composite-rigid-body inertia about the hinge axis
  plus armature), computed here with our own composite-inertia pass.
* foot contact spheres from the ``foot`` default class (gen_model.py:34-50)
* the ``stand`` keyframe                              (gen_model.py:141)

Outputs (both committed):
  g1sim_b200/model/g1_model_data.py   -- numpy-free Python literals
  g1sim_b200/csrc/g1_model_data.h     -- C/C++ constant tables (double)
  g1sim_b200/csrc/g1_model_derived.h  -- derived tables for the device code

Usage:  python g1sim_b200/model/gen_model.py <dir containing g1_stripped.xml and g1_raw.xml>
"""
import math
import os
import sys
import xml.etree.ElementTree as ET

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)

# The reference's checked-in header runs with mu = 1.0 (src/g1_model.h:351),
# although the foot class of model/g1_raw.xml says friction="0.6".  The value
# that the reference's code actually uses is the one kept here.
CONTACT_MU = 1.0
SINCOS_K = 202


def _vec(s, n=None):
    v = [float(x) for x in s.split()]
    if n is not None:
        assert len(v) == n, (s, n)
    return v


def quat_normalize(q):
    q = np.asarray(q, dtype=np.float64)
    n = math.sqrt(float(q @ q))
    return q / n


def quat_to_mat(q):
    """Rotation matrix of a unit quaternion (w, x, y, z), row-major 3x3.

    Standard formula written with the squared terms of all four components so
    that a unit quaternion maps to an orthonormal matrix to rounding.
    """
    w, x, y, z = (float(c) for c in q)
    if w == 1.0 and x == 0.0 and y == 0.0 and z == 0.0:
        return np.eye(3)
    ww, xx, yy, zz = w * w, x * x, y * y, z * z
    wx, wy, wz = w * x, w * y, w * z
    xy, xz, yz = x * y, x * z, y * z
    return np.array([
        [ww + xx - yy - zz, 2 * (xy - wz), 2 * (xz + wy)],
        [2 * (xy + wz), ww - xx + yy - zz, 2 * (yz - wx)],
        [2 * (xz - wy), 2 * (yz + wx), ww - xx - yy + zz],
    ])


def parse(model_dir):
    stripped = ET.parse(os.path.join(model_dir, "g1_stripped.xml")).getroot()
    raw = ET.parse(os.path.join(model_dir, "g1_raw.xml")).getroot()

    # defaults of class g1 (joint armature, position kp / dampratio)
    armature_default, damping_default = 0.0, 0.0
    kp_default, dampratio_default = None, None
    for d in stripped.iter("default"):
        if d.get("class") == "g1":
            j = d.find("joint")
            if j is not None:
                armature_default = float(j.get("armature", 0.0))
                damping_default = float(j.get("damping", 0.0))
            p = d.find("position")
            if p is not None:
                kp_default = float(p.get("kp"))
                dampratio_default = float(p.get("dampratio", 0.0))
    assert kp_default is not None

    bodies = []  # dicts, document (depth-first) order

    def walk(el, parent):
        for b in el.findall("body"):
            inert = b.find("inertial")
            rec = {
                "name": b.get("name"),
                "parent": parent,
                "pos": _vec(b.get("pos", "0 0 0"), 3),
                "quat": list(quat_normalize(_vec(b.get("quat", "1 0 0 0"), 4))),
                "mass": float(inert.get("mass")),
                "ipos": _vec(inert.get("pos"), 3),
                "iquat": list(quat_normalize(_vec(inert.get("quat", "1 0 0 0"), 4))),
                "diag": _vec(inert.get("diaginertia"), 3),
            }
            j = b.find("joint")
            fj = b.find("freejoint")
            if fj is not None:
                rec["joint"] = "free"
            else:
                assert j is not None, rec["name"]
                rec["joint"] = "hinge"
                rec["jname"] = j.get("name")
                rec["axis"] = list(np.asarray(_vec(j.get("axis", "0 0 1"), 3))
                                   / np.linalg.norm(_vec(j.get("axis", "0 0 1"), 3)))
                rec["anchor"] = _vec(j.get("pos", "0 0 0"), 3)
                rec["range"] = _vec(j.get("range"), 2)
                rec["frclim"] = abs(_vec(j.get("actuatorfrcrange"), 2)[1])
                rec["armature"] = float(j.get("armature", armature_default))
                rec["damping"] = float(j.get("damping", damping_default))
            idx = len(bodies)
            bodies.append(rec)
            walk(b, idx)

    walk(stripped.find("worldbody"), -1)
    assert bodies[0]["joint"] == "free"
    nb = len(bodies)

    # actuators: one position servo per hinge, in hinge order
    acts = [a.get("joint") for a in stripped.find("actuator").findall("position")]
    hinge_names = [b["jname"] for b in bodies[1:]]
    assert acts == hinge_names, "actuator order must match the hinge order"

    # foot spheres from the raw model
    foot_radius = None
    for d in raw.iter("default"):
        if d.get("class") == "foot":
            foot_radius = float(d.find("geom").get("size"))
    name_to_idx = {b["name"]: i for i, b in enumerate(bodies)}
    cbody, cpos = [], []
    for b in raw.iter("body"):
        for g in b.findall("geom"):
            if g.get("class") == "foot":
                cbody.append(name_to_idx[b.get("name")])
                cpos.append(_vec(g.get("pos"), 3))
    assert len(cbody) == 8

    key = stripped.find("keyframe").find("key")
    qpos_stand = _vec(key.get("qpos"))
    return bodies, nb, kp_default, dampratio_default, foot_radius, cbody, cpos, qpos_stand


def composite_diag(bodies, icom):
    """Joint-space mass-matrix diagonal of each hinge at qpos0 (all hinges 0).

    At qpos0 every body frame sits at its tree pose, so the composite inertia
    of the subtree of body i, expressed in body i's frame, accumulates
    leaf-to-root with the tree transforms only.  M0[h] = S^T Ic S + armature.
    """
    nb = len(bodies)
    # spatial inertia of each body at its own origin: [ang; lin] 6x6
    I = []
    for i, b in enumerate(bodies):
        m = b["mass"]
        c = np.asarray(b["ipos"])
        cx = np.array([[0, -c[2], c[1]], [c[2], 0, -c[0]], [-c[1], c[0], 0]])
        S = np.zeros((6, 6))
        S[:3, :3] = icom[i] + m * cx @ cx.T
        S[:3, 3:] = m * cx
        S[3:, :3] = m * cx.T
        S[3:, 3:] = m * np.eye(3)
        I.append(S)
    Ic = [x.copy() for x in I]
    for i in range(nb - 1, 0, -1):
        b = bodies[i]
        R = quat_to_mat(b["quat"])
        p = np.asarray(b["pos"])
        px = np.array([[0, -p[2], p[1]], [p[2], 0, -p[0]], [-p[1], p[0], 0]])
        # force transform child -> parent: [[R, p x R], [0, R]]
        Xf = np.zeros((6, 6))
        Xf[:3, :3] = R
        Xf[:3, 3:] = px @ R
        Xf[3:, 3:] = R
        Ic[b["parent"]] += Xf @ Ic[i] @ Xf.T
    m0 = []
    for i in range(1, nb):
        b = bodies[i]
        ax = np.asarray(b["axis"])
        an = np.asarray(b["anchor"])
        S = np.concatenate([ax, np.cross(an, ax)])
        m0.append(float(S @ Ic[i] @ S) + b["armature"])
    return m0


def build(model_dir):
    bodies, nb, kp, dampratio, radius, cbody, cpos, qpos_stand = parse(model_dir)
    icom = []
    for b in bodies:
        R = quat_to_mat(b["iquat"])
        icom.append(R @ np.diag(b["diag"]) @ R.T)
    m0 = composite_diag(bodies, icom)
    hinges = bodies[1:]
    data = {
        "NB": nb,
        "NV": 6 + len(hinges),
        "NQ": 7 + len(hinges),
        "NU": len(hinges),
        "NC": len(cbody),
        "body_names": [b["name"] for b in bodies],
        "parent": [b["parent"] for b in bodies],
        "tree_pos": [list(map(float, b["pos"])) for b in bodies],
        "tree_quat": [list(map(float, b["quat"])) for b in bodies],
        "mass": [b["mass"] for b in bodies],
        "com": [list(map(float, b["ipos"])) for b in bodies],
        "inertia_com": [list(map(float, x.reshape(-1))) for x in icom],
        "jnt_axis": [list(map(float, b["axis"])) for b in hinges],
        "jnt_anchor": [list(map(float, b["anchor"])) for b in hinges],
        "armature": [b["armature"] for b in hinges],
        "damping": [b["damping"] for b in hinges],
        "jnt_range": [list(map(float, b["range"])) for b in hinges],
        "act_kp": [kp] * len(hinges),
        "act_kv": [2.0 * dampratio * math.sqrt(kp * m) for m in m0],
        "act_frclim": [b["frclim"] for b in hinges],
        "contact_body": cbody,
        "contact_pos": [list(map(float, p)) for p in cpos],
        "contact_radius": radius,
        "contact_mu": CONTACT_MU,
        "qpos_stand": qpos_stand,
    }
    return data


def _fmt(v):
    return repr(float(v))


def emit_py(data, path):
    with open(path, "w") as f:
        f.write("# Generated by g1sim_b200/model/gen_model.py from the G1 MJCF -- do not edit.\n")
        f.write("# Unitree G1 29-DoF (mujoco_menagerie g1_29dof_rev_1_0, stripped).\n")
        for k, v in data.items():
            f.write(f"{k} = {v!r}\n")


def emit_h(data, path):
    def arr(name, rows, ctype="double"):
        flat = []
        for r in rows:
            flat.extend(r if isinstance(r, (list, tuple)) else [r])
        if ctype == "int":
            body = ", ".join(str(int(x)) for x in flat)
        else:
            body = ",\n  ".join(", ".join(_fmt(x) for x in flat[i:i + 6])
                                for i in range(0, len(flat), 6))
        return f"G1M_TABLE {ctype} {name}[{len(flat)}] = {{\n  {body}\n}};\n"

    with open(path, "w") as f:
        f.write("// Generated by g1sim_b200/model/gen_model.py from the G1 MJCF -- do not edit.\n")
        f.write("// Unitree G1 29-DoF (mujoco_menagerie g1_29dof_rev_1_0, stripped).\n")
        f.write("// Plain C / C++ / CUDA: the tables are host constants; device code\n")
        f.write("// reads them only in constant expressions or copies them to __constant__.\n")
        f.write("#ifndef G1M_MODEL_DATA_H\n#define G1M_MODEL_DATA_H\n\n")
        f.write("#ifdef __cplusplus\n#define G1M_TABLE static constexpr\n#else\n"
                "#define G1M_TABLE static const\n#endif\n\n")
        for k in ("NB", "NV", "NQ", "NU", "NC"):
            f.write(f"#define G1M_{k} {data[k]}\n")
        f.write("\n// bodies: " + ", ".join(f"{i}:{n}" for i, n in enumerate(data["body_names"])) + "\n")
        f.write(arr("g1m_parent", data["parent"], "int"))
        for k in ("tree_pos", "tree_quat", "mass", "com", "inertia_com", "jnt_axis",
                  "jnt_anchor", "armature", "damping", "jnt_range", "act_kp", "act_kv",
                  "act_frclim"):
            f.write(arr("g1m_" + k, data[k]))
        f.write(arr("g1m_contact_body", data["contact_body"], "int"))
        f.write(arr("g1m_contact_pos", data["contact_pos"]))
        f.write(f"G1M_TABLE double g1m_contact_radius = {_fmt(data['contact_radius'])};\n")
        f.write(f"G1M_TABLE double g1m_contact_mu = {_fmt(data['contact_mu'])};\n")
        f.write(arr("g1m_qpos_stand", data["qpos_stand"]))
        f.write("\n#endif  // G1M_MODEL_DATA_H\n")


def derived(data):
    """Tables the device code uses directly (computed once, in double)."""
    nb = data["NB"]
    tree_rot, tree_ident, sp_inertia, axis_idx = [], [], [], []
    for i in range(nb):
        q = data["tree_quat"][i]
        ident = q == [1.0, 0.0, 0.0, 0.0]
        tree_ident.append(1 if ident else 0)
        tree_rot.append(list(map(float, quat_to_mat(q).reshape(-1))))
        m = data["mass"][i]
        c = np.asarray(data["com"][i])
        icom = np.asarray(data["inertia_com"][i]).reshape(3, 3)
        cx = np.array([[0, -c[2], c[1]], [c[2], 0, -c[0]], [-c[1], c[0], 0]])
        J = icom + m * cx @ cx.T          # about the body origin
        H = m * cx                        # angular-linear block
        # J (xx, yy, zz, xy, xz, yz), H row-major, M = m I
        sp_inertia.append([J[0, 0], J[1, 1], J[2, 2], J[0, 1], J[0, 2], J[1, 2]]
                          + list(H.reshape(-1)) + [m])
    # leg bodies: their tree rotation must be identity or a pure rotation
    # about y (the device composes it in extended precision as a (cos, sin)
    # pair); record cos / sin of that rotation
    tree_ycs = []
    for i in range(nb):
        R = np.asarray(tree_rot[i]).reshape(3, 3)
        if tree_ident[i]:
            tree_ycs.append([1.0, 0.0])
            continue
        is_y = abs(R[1, 1] - 1) < 1e-15 and abs(R[0, 1]) < 1e-15 and abs(R[1, 0]) < 1e-15 \
            and abs(R[1, 2]) < 1e-15 and abs(R[2, 1]) < 1e-15
        leg = 1 <= i <= 12
        assert is_y or not leg, f"leg body {i}: tree rotation is not about y"
        q = data["tree_quat"][i]
        ang = 2.0 * math.atan2(q[2], q[0]) if is_y else 0.0
        tree_ycs.append([math.cos(ang), math.sin(ang)] if is_y else [1.0, 0.0])
    for h, ax in enumerate(data["jnt_axis"]):
        nz = [k for k in range(3) if ax[k] != 0.0]
        assert len(nz) == 1 and ax[nz[0]] == 1.0, "hinge axes must be +x, +y or +z"
        assert data["jnt_anchor"][h] == [0.0, 0.0, 0.0], "hinge anchors must be at the body origin"
        axis_idx.append(nz[0])
    # sin / cos of k / 32 rad for |k| <= 202 (|angle| <= 6.3125), in double, for
    # the device's extended-precision sin/cos (angle addition + short Taylor).
    sincos_tab = []
    for k in range(-SINCOS_K, SINCOS_K + 1):
        a = k / 32.0
        sincos_tab.append([math.sin(a), math.cos(a)])
    return dict(tree_rot=tree_rot, tree_ident=tree_ident, sp_inertia=sp_inertia,
                axis_idx=axis_idx, sincos_tab=sincos_tab, tree_ycs=tree_ycs)


def emit_derived_h(data, der, path):
    def arr(name, rows, ctype="double"):
        flat = []
        for r in rows:
            flat.extend(r if isinstance(r, (list, tuple)) else [r])
        if ctype == "int":
            body = ", ".join(str(int(x)) for x in flat)
        else:
            body = ",\n  ".join(", ".join(_fmt(x) for x in flat[i:i + 6])
                                for i in range(0, len(flat), 6))
        return f"G1M_TABLE {ctype} {name}[{len(flat)}] = {{\n  {body}\n}};\n"

    with open(path, "w") as f:
        f.write("// Generated by g1sim_b200/model/gen_model.py -- do not edit.\n")
        f.write("// Derived G1 tables in double: tree rotation matrices (row-major, from\n")
        f.write("// the unit tree quaternions), rigid-body spatial inertia about each body\n")
        f.write("// origin as J(xx,yy,zz,xy,xz,yz), H = m [c]x (row-major), m, and the\n")
        f.write("// hinge axis index (every axis is +x, +y or +z, every anchor is 0).\n")
        f.write("#ifndef G1M_MODEL_DERIVED_H\n#define G1M_MODEL_DERIVED_H\n")
        f.write('#include "g1_model_data.h"\n\n')
        f.write(arr("g1m_tree_rot", der["tree_rot"]))
        f.write(arr("g1m_tree_ident", der["tree_ident"], "int"))
        f.write(arr("g1m_sp_inertia", der["sp_inertia"]))
        f.write(arr("g1m_axis_idx", der["axis_idx"], "int"))
        f.write(arr("g1m_tree_ycs", der["tree_ycs"]))
        f.write(f"#define G1M_SINCOS_K {SINCOS_K}\n")
        f.write(arr("g1m_sincos_tab", der["sincos_tab"]))
        f.write("\n#endif  // G1M_MODEL_DERIVED_H\n")


def main():
    model_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("G1_MJCF_DIR")
    if not model_dir:
        sys.exit("usage: gen_model.py <dir with g1_stripped.xml and g1_raw.xml>")
    data = build(model_dir)
    emit_py(data, os.path.join(HERE, "g1_model_data.py"))
    emit_h(data, os.path.join(PKG, "csrc", "g1_model_data.h"))
    emit_derived_h(data, derived(data), os.path.join(PKG, "csrc", "g1_model_derived.h"))
    print(f"NB={data['NB']} NV={data['NV']} NQ={data['NQ']} NU={data['NU']} NC={data['NC']}")


if __name__ == "__main__":
    main()
