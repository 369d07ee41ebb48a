"""Extracts the known answers that pin the steady Euler path from the
reference's own test files (read as text; nothing of the reference runs) into
reference_known_answers.json. Run from the repository root with the path of
a checkout of the reference, as an argument or in the REFERENCE variable:

    python tests/golden/extract_known_answers.py <reference checkout>

The tests read only the JSON file."""
from __future__ import annotations

import json
import os
import re
import sys
from pathlib import Path

def reference_root() -> Path:
    """The reference checkout: the first argument, else REFERENCE."""
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE")
    if not where:
        sys.exit("usage: extract_known_answers.py <reference checkout> (or set REFERENCE)")
    return Path(where)


REF = Path()
OUT = Path(__file__).resolve().parent / "reference_known_answers.json"


def find_line(text: str, needle: str) -> int:
    for k, line in enumerate(text.splitlines(), 1):
        if needle in line:
            return k
    raise KeyError(needle)


def main() -> None:
    global REF
    REF = reference_root()
    out: dict = {}
    # Verified drag of the CPU engine on the 20 deg cone at Mach 3 (cylinder 4,
    # nj = 20), refinements 1 and 2.
    f = "tests/gpu/verified-drag-gpu.test.ts"
    t = (REF / f).read_text()
    m = re.search(r"const cpu = \[([0-9.]+),\s*([0-9.]+)\]", t)
    out["verified_drag_cone20_mach3"] = {
        "source": f"{f}:{find_line(t, 'const cpu = [')}",
        "body": {"shape": "conical", "half_angle_deg": 20, "base_radius": 0.5, "cylinder": 4},
        "mach": 3.0, "nj": 20, "refinements": [1, 2],
        "drag": [float(m.group(1)), float(m.group(2))],
        "tolerance_relative": 2e-6,
    }
    # Taylor-Maccoll against NASA SP-3004 (cone deg, Mach, shock angle rad,
    # surface Mach, Cp) and the NPARC 10 deg / Mach 2.35 case.
    f = "tests/validation/taylor-maccoll.test.ts"
    t = (REF / f).read_text()
    rows = re.findall(r"\[\s*([0-9.]+),\s*([0-9.]+),\s*([0-9.]+),\s*([0-9.]+),\s*([0-9.]+)\s*\]", t)
    out["taylor_maccoll_sp3004"] = {
        "source": f"{f}:{find_line(t, 'const rows')}",
        "columns": ["cone_deg", "mach", "shock_angle_rad", "surface_mach", "cp"],
        "rows": [[float(v) for v in r] for r in rows],
        "tolerance": {"shock_angle_abs": 5e-6, "surface_mach_rel": 3e-5, "cp_abs": 3e-5},
    }
    # Grid-convergence families measured on cone-cylinders (mean cone
    # surface pressure over the free stream's on nj = 20, 40, 80, 160) with
    # their Taylor-Maccoll values, and the options the reference checks
    # their bands with.
    fg = "tests/verification/grid-convergence.test.ts"
    tg = (REF / fg).read_text()
    fams = re.findall(r"\['([^']+)',\s*([0-9.]+),\s*\[([0-9.,\s]+)\]\]", tg)
    out["grid_convergence_cone_families"] = {
        "source": f"{fg}:{find_line(tg, 'const families')}",
        "options": {"order_tolerance": 0.5, "noise": 1e-12, "floor": 2e-4, "max_refinement": 8},
        "families": [{"name": name, "exact": float(exact), "values": [float(v) for v in vals.split(",")]}
                     for name, exact, vals in fams],
    }
    out["taylor_maccoll_nparc"] = {
        "source": f"{f}:{find_line(t, 'NPARC/WIND')}",
        "cone_deg": 10, "mach": 2.35,
        "post_shock_mach": 2.2677, "surface_mach": 2.1469, "surface_mach_cfd": 2.1467886,
        "surface_pressure_ratio": 1.37405,
        "tolerance": {"post_shock_mach_abs": 5e-4, "surface_mach_abs": 5e-4,
                      "surface_mach_cfd_abs": 2e-4, "surface_pressure_ratio_abs": 5e-4},
    }
    assert re.search(r"toBeCloseTo\(2\.2677", t) is not None
    # Implicit steps reach the explicit drag (15 deg cone, Mach 2, nj 12, cylinder 1).
    f = "tests/engine-cpu/implicit.test.ts"
    t = (REF / f).read_text()
    out["implicit_equals_explicit"] = {
        "source": f"{f}:{find_line(t, 'implicit steps reach the steady state')}",
        "body": {"shape": "conical", "half_angle_deg": 15, "base_radius": 0.5, "cylinder": 1},
        "mach": 2.0, "nj": 12, "explicit_steps": 6000, "residual_below": 1e-12,
        "drag_equal_within": 1e-12,
    }
    # Anderson acceleration (src/solver/anderson.ts): its own known answers,
    # and the accelerated LU-SGS steps on the same cone.
    plain = re.search(r"new AndersonMixing\(3, (\d+)\);\s*const x = Float64Array\.from\(\[([^\]]*)\]\);"
                      r"\s*const f = Float64Array\.from\(\[([^\]]*)\]\);\s*"
                      r"expect\(Array\.from\(a\.next\(x, f\)\)\)\.toEqual\(\[([^\]]*)\]\)", t)
    linear = re.search(r"const n = (\d+);\s*const diag = .*?1 / \(1 \+ \((\d+) \* k\) / \(n - 1\)\)\).*?"
                       r"new AndersonMixing\(n, (\d+)\);\s*for \(let k = 0; k < (\d+); k\+\+\).*?"
                       r"toBeLessThan\(([0-9e.-]+) \* error.*?toBeGreaterThan\(([0-9.]+) \* error", t, re.S)
    lusgs = re.search(r"s\.iterateImplicit\((\d+), (\d+)\);\s*const n = 4 \* grid\.ni \* grid\.nj;\s*"
                      r"const anderson = new AndersonMixing\(n, (\d+)\);\s*for \(let k = 0; k < (\d+) .*?"
                      r"implicitCorrection\((\d+)\)", t, re.S)
    nums = lambda g: [float(v) for v in g.split(",")]
    out["anderson"] = {
        "source": f"{f}:{find_line(t, 'without history takes the plain step')}",
        "plain_step": {"depth": int(plain.group(1)), "x": nums(plain.group(2)), "f": nums(plain.group(3)),
                       "next": nums(plain.group(4))},
        "linear": {"n": int(linear.group(1)), "stiffness": int(linear.group(2)), "depth": int(linear.group(3)),
                   "steps": int(linear.group(4)), "accelerated_below": float(linear.group(5)),
                   "plain_above": float(linear.group(6)),
                   "correction": "(b - diag x) / 4, diag_k = 1 / (1 + stiffness k / (n - 1)), b_k = sin(k + 1)"},
        "lusgs": {"source": f"{f}:{find_line(t, 'Anderson-accelerated LU-SGS gives the same drag')}",
                  "plain_steps": int(lusgs.group(1)), "plain_cfl": float(lusgs.group(2)),
                  "depth": int(lusgs.group(3)), "max_steps": int(lusgs.group(4)), "cfl": float(lusgs.group(5)),
                  "residual_below": 1e-12, "drag_equal_within": 1e-12},
    }
    # The fitted bow shock on the Mach 3, 20 deg cone (cylinder 4): the drag's
    # error against Taylor-Maccoll measured when the reference's test was
    # written, and the bounds the test asserts.
    f = "tests/analysis/fitted-flow.test.ts"
    t = (REF / f).read_text()
    m = re.search(r"Measured when\s*//\s*written: \+([0-9.]+)% on 10 cells across, \+([0-9.]+)% on that grid", t)
    bounds = re.search(r"expect\(Math\.abs\(fine\)\)\.toBeLessThan\(([0-9e.-]+)\);\s*"
                       r"expect\(coarse / fine\)\.toBeGreaterThan\(([0-9.]+)\);\s*"
                       r"expect\(coarse / fine\)\.toBeLessThan\(([0-9.]+)\);\s*"
                       r"expect\(Math\.abs\(fine - \(coarse - fine\) / 3\)\)\.toBeLessThan\(([0-9e.-]+)\)", t)
    out["fitted_cone_mach3"] = {
        "source": f"{f}:{find_line(t, 'Mach 3, 20 deg cone: drag within')}",
        "body": {"shape": "conical", "half_angle_deg": 20, "base_radius": 0.5, "cylinder": 4},
        "mach": 3.0, "nj": 10, "refinements": [1, 2],
        "measured_rel_err": [float(m.group(1)) / 100, float(m.group(2)) / 100],
        "fine_below": float(bounds.group(1)), "ratio_above": float(bounds.group(2)),
        "ratio_below": float(bounds.group(3)), "extrapolated_within": float(bounds.group(4)),
    }
    hm = re.search(r"Measured when written: \+([0-9.]+)% \(nj = (\d+)\); with the captured shock \+([0-9.]+)%", t)
    tol = re.search(r"expect\(Math\.abs\(p / pitot - 1\)\)\.toBeLessThan\(([0-9e.-]+)\)", t)
    out["fitted_hemisphere_mach2"] = {
        "source": f"{f}:{find_line(t, 'Mach 2 hemisphere-cylinder')}",
        "body": {"shape": "ellipsoid", "length": 0.5, "base_radius": 0.5, "cylinder": 4},
        "mach": 2.0, "nj": int(hm.group(2)),
        "measured_rel_err": float(hm.group(1)) / 100, "captured_rel_err": float(hm.group(3)) / 100,
        "within": float(tol.group(1)),
    }
    # The 3-caliber tangent ogive: at Mach 1.35 (axially subsonic tip) the
    # page's family and its coarser one; at Mach 1.5 on 30 calibers of
    # cylinder the fallback to more columns.
    fam = re.search(r"nj = 20 to 160.*?converged to 1e-10 of its drag\):\s*([0-9.]+), ([0-9.]+),\s*//\s*([0-9.]+), "
                    r"([0-9.]+), at orders.*?extrapolated\s*//\s*to ([0-9.]+)", t, re.S)
    coarse = re.search(r"\+([0-9.e-]+) and \+([0-9.e-]+) of that value, falling by ([0-9]+\.[0-9]+)", t)
    ob = re.search(r"expect\(fine\)\.toBeLessThan\(([0-9e.-]+)\);\s*expect\(coarse / fine\)\.toBeGreaterThan\(([0-9.]+)\);"
                   r"\s*expect\(coarse / fine\)\.toBeLessThan\(([0-9.]+)\);", t)
    base = re.search(r"expect\(result\.levels\[0\]!\.value\)\.toBe\(([0-9.]+)\)", t)
    out["fitted_ogive_mach1_35"] = {
        "source": f"{f}:{find_line(t, 'Mach 1.35, 3-caliber tangent ogive')}",
        "body": {"shape": "ogive", "parameter": 1, "length": 3, "base_radius": 0.5, "cylinder": 2},
        "mach": 1.35, "family_nj20": [float(fam.group(k)) for k in range(1, 5)],
        "extrapolated": float(fam.group(5)),
        "coarse_family_nj10_rel": [float(coarse.group(1)), float(coarse.group(2))],
        "coarse_family_ratio": float(coarse.group(3)),
        "fine_below": float(ob.group(1)), "ratio_above": float(ob.group(2)), "ratio_below": float(ob.group(3)),
        "verified_nj20_value": float(base.group(1)),
    }
    fb = re.search(r"aspect ratio of ([0-9.]+) \(measured\s*//\s*when written\), above the (\d+) allowed", t)
    fv = re.search(r"Measured when written: ([0-9.]+) on (\d+) columns", t)
    out["fitted_ogive_fallback_mach1_5"] = {
        "source": f"{f}:{find_line(t, 'a sharp nose whose usual grid fails only the quality gates')}",
        "body": {"shape": "ogive", "parameter": 1, "length": 3, "base_radius": 0.5, "cylinder": 30},
        "mach": 1.5, "aspect_ratio": float(fb.group(1)), "aspect_limit": int(fb.group(2)),
        "value": float(fv.group(1)), "columns": int(fv.group(2)), "equal_within": 1e-12,
    }
    # A two-scale family on the CPU engine: the 1-caliber Von Karman nose
    # with a caliber of body at Mach 2, its fitted drags on nj = 20 and 40.
    f2 = "tests/analysis/two-scale-fit.test.ts"
    t2 = (REF / f2).read_text()
    meas = re.search(r"const MEASURED = \[([0-9.]+), ([0-9.]+)\];", t2)
    vk = re.search(r"shape: \{ kind: 'haack', parameter: 0 \}, length: ([0-9.]+), baseRadius: ([0-9.]+) \},\s*"
                   r"cylinderLength: ([0-9.]+),", t2)
    opts = re.search(r"const familyOptions = \{ mach: ([0-9.]+), gamma, nj: (\d+) \};", t2)
    out["fitted_von_karman_mach2"] = {
        "source": f"{f2}:{find_line(t2, 'const MEASURED')}",
        "body": {"shape": "haack", "parameter": 0, "length": float(vk.group(1)),
                 "base_radius": float(vk.group(2)), "cylinder": float(vk.group(3))},
        "mach": float(opts.group(1)), "nj": int(opts.group(2)),
        "drag_nj20": float(meas.group(1)), "drag_nj40": float(meas.group(2)), "within": 1e-9,
    }
    # Transonic flow: the 7 deg cone of NACA TN 4233 at Mach 1.2 on its
    # transonic grids, the drags measured on the base grid and the next two.
    f3 = "tests/analysis/transonic-flow.test.ts"
    t3 = (REF / f3).read_text()
    tn = (REF / "src/validation/cone-cylinder-tn4233.ts").read_text()
    half = re.search(r"TN4233_CONE_HALF_ANGLE = \(\(([0-9]+) \+ ([0-9]+) / 60\) \* Math\.PI\) / 180;", tn)
    m3 = re.search(r"Measured when\s*//\s*written: ([0-9.]+) on the base grid \(\+([0-9.]+)%\), ([0-9.]+) and\s*//\s*"
                   r"([0-9.]+) on the next two", t3)
    po = re.search(r"mach: ([0-9.]+),\s*gamma,\s*refinement: 1,\s*farField: ([0-9]+),\s*cylinder: ([0-9]+),", t3)
    so = re.search(r"noise: ([0-9e.-]+),\s*maxSteps: ([0-9]+),\s*checkEvery: ([0-9]+),\s*cfl: ([0-9]+),\s*"
                   r"depth: ([0-9]+),\s*plainSteps: ([0-9]+),", t3)
    within = re.search(r"toBeLessThan\(([0-9e.-]+)\);", t3)
    out["transonic_cone_tn4233_mach1_2"] = {
        "source": f"{f3}:{find_line(t3, 'Measured when')}",
        "cone_half_angle_deg": int(half.group(1)) + int(half.group(2)) / 60, "base_radius": 1.0,
        "mach": float(po.group(1)), "far_field": float(po.group(2)), "cylinder": float(po.group(3)),
        "solve": {"noise": float(so.group(1)), "max_steps": int(so.group(2)), "check_every": int(so.group(3)),
                  "cfl": float(so.group(4)), "depth": int(so.group(5)), "plain_steps": int(so.group(6))},
        "drags": [float(m3.group(1)), float(m3.group(3)), float(m3.group(4))],
        "base_rel_vs_taylor_maccoll": float(m3.group(2)) / 100, "within_taylor_maccoll": float(within.group(1)),
    }
    # The two-scale allowance (TWO_SCALE_DRAG_FLOOR).
    fv2 = "src/analysis/verified-drag.ts"
    tf = (REF / fv2).read_text()
    floor = re.search(r"export const TWO_SCALE_DRAG_FLOOR = ([0-9.e-]+);", tf)
    out["two_scale_drag_floor"] = {"source": f"{fv2}:{find_line(tf, 'export const TWO_SCALE_DRAG_FLOOR')}",
                                   "value": float(floor.group(1))}
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    sys.exit(main())
