"""Writes the golden fixtures of tests/golden from the reference itself.

Run in a checkout that has the reference's sources (its Python package
`precomp` imports without a build): ``python tests/golden/make_golden.py
<reference root>``. The fixtures it writes are committed; the tests read
only them, never the reference.

strip_h2_im_nz4.json, strip_h1_im_nz4.json, plate_h2_im_mu0.1_drag3.json
(incompatible-mode Hex8) and strip_h2_std_mu0.1.json,
plate_h2_std_mu0.1_drag3.json (standard Hex8 with mean dilatation),
strip_h2_nobbar_mu0.1.json (standard Hex8 without): committed forming runs
of the reference (benchmarks/physics_audit/calculix/punch/<case>/sparlab):
the mesh, the parts of its deck the element loop and the contact read
(material, model and element formulation, mean dilatation, kinematics,
tool, steps and their boundary regions), the nodal
displacements at the end of each step (17 significant digits in the
reference's CSV output), the step-end element fields (largest equivalent
plastic strain of the element's points, von Mises stress of its averaged
Cauchy stress) and the tool force of every forming increment.

kin_h0833.json + kin_h0833.npz: the reference's forming run
benchmarks/physics_audit/challenge/cases/kin_h0833 - a 48 x 48 x 1
incompatible-mode sheet with the 2 x 2 x 5 rule, Hill48 with two Chaboche
backstresses and Voce hardening, a spherical tool on a 113-knot spiral
path - the deck's parts in the JSON (the tool path read from its CSV), the
mesh, the step-end displacements and element fields in the npz.

parts.json: heights of the reference's part families at sample points.

materials.json: the hardening parameters the reference's own Python
(python/precomp/materials.py) derives - its built-in library (Hollomon
fits) and the Swift law of the 40x40x2 forming sheet - plus the material
blocks of the committed forming decks under benchmarks/ that the
reference's C++ runs read.
"""
from __future__ import annotations

import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
KEYS = ("youngs_modulus", "poisson_ratio", "yield_stress", "hardening_modulus", "saturation_stress",
        "saturation_rate", "kinematic_hardening_modulus")


def main(ref_root: str) -> None:
    sys.path.insert(0, os.path.join(ref_root, "python"))
    from precomp import materials  # the reference's own module

    out = {"library": {}, "swift": [], "decks": {}}
    for name, m in sorted(materials.library().items()):
        out["library"][name] = {k: getattr(m, k) for k in KEYS}
    for K, eps0, n in [(425e6, 0.003, 0.29), (530e6, 0.005, 0.22), (600e6, 0.01, 0.15)]:
        m = materials.Material.from_swift("swift", 70e9, 0.33, 2700.0, K=K, eps0=eps0, n=n)
        out["swift"].append({"K": K, "eps0": eps0, "n": n, **{k: getattr(m, k) for k in KEYS}})
    for deck in sorted(glob.glob(os.path.join(ref_root, "benchmarks/physics_audit/calculix/punch/strip_h*_im_*/"
                                                       "sparlab/deck.json")))[:4]:
        d = json.load(open(deck))
        mat = d["material"]
        rel = os.path.relpath(deck, ref_root)
        out["decks"][rel] = {"name": mat["name"], "youngs_modulus": mat["youngs_modulus"],
                             "poisson_ratio": mat["poisson_ratio"], **mat["plasticity"]}
    with open(os.path.join(HERE, "materials.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


def strip(ref_root: str, case: str = "strip_h2_im_nz4") -> None:
    import csv

    base = os.path.join(ref_root, "benchmarks/physics_audit/calculix/punch", case, "sparlab")
    deck = json.load(open(os.path.join(base, "deck.json")))
    mesh = json.load(open(os.path.join(base, "out", "mesh.json")))
    summary = json.load(open(os.path.join(base, "out", "summary.json")))
    steps = []
    for k, st in enumerate(deck["forming"]["steps"], start=1):
        rows = list(csv.DictReader(open(os.path.join(base, "out", f"step_{k}_{st['name']}_nodes.csv"))))
        steps.append({"deck": st, "u": [[float(r["ux"]), float(r["uy"]), float(r["uz"])] for r in rows],
                      "increments": summary["steps"][k - 1]["increments"],
                      "cuts": summary["steps"][k - 1]["cuts"],
                      "elements": element_fields(os.path.join(base, "out"), k, st["name"])})
    forces = [{k: r[k] for k in ("step", "increment", "t", "cx", "cz", "fx", "fz", "active_nodes")}
              for r in csv.DictReader(open(os.path.join(base, "out", "tool_forces.csv")))]
    out = {"source": os.path.relpath(base, ref_root), "nodes": mesh["nodes_m"], "elements": mesh["elements"],
           "material": deck["material"], "model": deck.get("model", {}),
           "mean_dilatation": deck["forming"].get("mean_dilatation", "auto"),
           "kinematics": deck["forming"]["kinematics"],
           "tools": deck["forming"]["tools"], "steps": steps, "tool_forces": forces,
           "analysis": summary["analysis"]}
    with open(os.path.join(HERE, f"{case}.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")


def element_fields(out_dir: str, k: int, name: str) -> dict:
    """The step-end element fields the reference writes
    (step_<k>_<s>_elements.csv: element, eq_plastic_strain, von_mises_Pa;
    include/sparlab/io/FormingWriter.hpp:1-12), in element order."""
    import csv

    rows = list(csv.DictReader(open(os.path.join(out_dir, f"step_{k}_{name}_elements.csv"))))
    assert [int(r["element"]) for r in rows] == list(range(len(rows)))
    return {"eq_plastic_strain": [float(r["eq_plastic_strain"]) for r in rows],
            "von_mises_Pa": [float(r["von_mises_Pa"]) for r in rows]}


def challenge(ref_root: str, case: str = "kin_h0833") -> None:
    import csv

    import numpy as np

    base = os.path.join(ref_root, "benchmarks/physics_audit/challenge/cases", case)
    deck = json.load(open(os.path.join(base, "deck", "deck.json")))
    mesh = json.load(open(os.path.join(base, "output", "mesh.json")))
    summary = json.load(open(os.path.join(base, "output", "summary.json")))
    tools = []
    for t in deck["forming"]["tools"]:
        t = dict(t)
        tr = t["trajectory"]
        if "file" in tr:
            rows = list(csv.DictReader(open(os.path.join(base, "deck", tr["file"]))))
            t["trajectory"] = {"times": [float(r["t"]) for r in rows],
                               "points": [[float(r["x"]), float(r["y"]), float(r["z"])] for r in rows]}
        tools.append(t)
    steps, us, eqps, vm = [], [], [], []
    for k, st in enumerate(deck["forming"]["steps"], start=1):
        rows = list(csv.DictReader(open(os.path.join(base, "output", f"step_{k}_{st['name']}_nodes.csv"))))
        us.append([[float(r["ux"]), float(r["uy"]), float(r["uz"])] for r in rows])
        fields = element_fields(os.path.join(base, "output"), k, st["name"])
        eqps.append(fields["eq_plastic_strain"])
        vm.append(fields["von_mises_Pa"])
        steps.append({"deck": st, "increments": summary["steps"][k - 1]["increments"],
                      "cuts": summary["steps"][k - 1]["cuts"]})
    forces = [{k: r[k] for k in ("step", "increment", "t", "cx", "cz", "fx", "fz", "active_nodes")}
              for r in csv.DictReader(open(os.path.join(base, "output", "tool_forces.csv")))]
    out = {"source": os.path.relpath(base, ref_root), "material": deck["material"], "model": deck["model"],
           "kinematics": deck["forming"]["kinematics"], "tools": tools, "steps": steps, "tool_forces": forces,
           "analysis": summary["analysis"], "arrays": case + ".npz"}
    with open(os.path.join(HERE, f"{case}.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    np.savez_compressed(os.path.join(HERE, f"{case}.npz"), nodes=np.array(mesh["nodes_m"], dtype=np.float64),
                        elements=np.array(mesh["elements"], dtype=np.int32), u=np.array(us, dtype=np.float64),
                        eq_plastic_strain=np.array(eqps, dtype=np.float64), von_mises=np.array(vm, dtype=np.float64))


def parts(ref_root: str) -> None:
    """parts.json: heights of the reference's four part families
    (python/precomp/geometry/parts.py) at seeded sample points, for a few
    parameter sets each - the cone of the fine-mesh configuration (18 mm
    footprint, 3 mm deep, 50 degree wall) among them."""
    import numpy as np

    sys.path.insert(0, os.path.join(ref_root, "python"))
    from precomp.geometry import parts as P  # the reference's own module

    cases = [
        ("truncated_cone", dict(top_radius=0.0093, wall_angle_deg=50.0, depth=0.003, top_fillet=0.001,
                                bottom_fillet=0.001)),
        ("truncated_cone", dict(top_radius=0.05, wall_angle_deg=35.0, depth=0.02, top_fillet=0.005,
                                bottom_fillet=0.004)),
        ("elliptic_cone", dict(semi_axis_x=0.009, semi_axis_y=0.007, wall_angle_deg=45.0, depth=0.0025,
                               top_fillet=0.001, bottom_fillet=0.001)),
        ("elliptic_cone", dict(semi_axis_x=0.05, semi_axis_y=0.06, wall_angle_deg=55.0, depth=0.015,
                               top_fillet=0.004, bottom_fillet=0.003)),
        ("pyramid", dict(half_width_x=0.009, half_width_y=0.0075, wall_angle_deg=40.0, depth=0.0025,
                         corner_radius=0.005, top_fillet=0.001, bottom_fillet=0.001)),
        ("dome", dict(opening_radius=0.009, depth=0.003, rim_fillet=0.002, aspect=1.0)),
        ("dome", dict(opening_radius=0.05, depth=0.02, rim_fillet=0.01, aspect=0.8)),
    ]
    rng = np.random.default_rng(1234)
    out = []
    for family, kw in cases:
        part = P.families()[family](**kw)
        r = 1.3 * part.footprint_radius()
        xy = rng.uniform(-r, r, size=(400, 2))
        xy[:8] = [[0, 0], [r / 2, 0], [0, r / 2], [r / 3, r / 4], [-r / 5, r / 7], [r, 0], [0, -r], [1e-6, 0]]
        z = part.height(xy[:, 0], xy[:, 1])
        out.append({"family": family, "params": kw, "footprint_radius": part.footprint_radius(),
                    "xy": xy.tolist(), "z": [float(v) for v in z]})
    with open(os.path.join(HERE, "parts.json"), "w") as f:
        json.dump(out, f)
        f.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the reference's checkout>")
    root = sys.argv[1]
    main(root)
    for case in ("strip_h2_im_nz4", "strip_h1_im_nz4", "plate_h2_im_mu0.1_drag3", "strip_h2_std_mu0.1",
                 "plate_h2_std_mu0.1_drag3", "strip_h2_nobbar_mu0.1"):
        strip(root, case)
    challenge(root)
    parts(root)
