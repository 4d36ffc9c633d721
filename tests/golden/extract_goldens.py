"""Extract the reference's bit-exact golden vectors into reference_goldens.json.

Reads crates/gemray/tests/raytracer_tests.rs of the reference checkout as TEXT (it is
never compiled or run) and records, with their source lines:
  * non_biaxial_materials_render_bit_identical_to_pre_chapter_04_golden_values
    (5 materials, XYZ as f32 bit patterns, raytracer_tests.rs:1374-1524);
  * studio_rig_refactor_is_bit_identical_to_pre_refactor_baseline: 4 traced cases x
    {Diamond, Sapphire}, 4 directions x 3 wavelengths of sample_studio_environment,
    and 5 evaluate_gem_optical_metrics bit patterns (raytracer_tests.rs:1627-1842).
Usage (in a checkout that has the reference): python extract_goldens.py <reference root>
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HEX = r"0x([0-9A-Fa-f_]+)"


def h(s: str) -> int:
    return int(s.replace("_", ""), 16)


def main(root: str) -> None:
    path = Path(root) / "crates/gemray/tests/raytracer_tests.rs"
    lines = path.read_text().splitlines()
    text = "\n".join(lines)
    out: dict = {"source": "crates/gemray/tests/raytracer_tests.rs"}

    # --- 5-material golden table
    start = text.index("let golden: &[(&str, u32, u32, u32)] = &[")
    end = text.index("];", start)
    block = text[start:end]
    mats = []
    for m in re.finditer(r'\(\s*"([^"]+)",\s*' + HEX + r",\s*" + HEX + r",\s*" + HEX, block, re.S):
        mats.append({"material": m.group(1), "xyz_bits": [h(m.group(2)), h(m.group(3)), h(m.group(4))]})
    out["materials"] = {
        "line": text[:start].count("\n") + 1,
        "ray_origin": [0.0, 2.5, 0.0], "ray_dir_unnormalized": [0.18, -1.0, 0.07],
        "seed": 1, "max_bounces": 12, "preset": "RingLights", "exposure": 1.0,
        "light_yaw": 0.85, "light_pitch": 0.95, "cases": mats,
    }

    # --- studio-rig traced cases
    start = text.index("let cases: [GoldenCase; 4] = [")
    end = text.index("];\n\n    for (ray, seed", start)
    block = text[start:end]
    case_re = re.compile(
        r"origin: Vec3::new\(([^)]*)\),\s*dir: Vec3::new\(([^)]*)\)(\.normalize\(\))?,\s*\},\s*(\d+),\s*"
        r"LightingPreset::(\w+),\s*([^,]+),\s*([^,]+),\s*\[([^\]]+)\],", re.S)
    cases = []
    for m in case_re.finditer(block):
        tail = block[m.end():]
        # the sapphire column is the last [..] before the closing paren of this case
        close = tail.index("),\n")
        sap = re.findall(r"\[(0x[^\]]+)\]", tail[:close])[-1]

        def nums(s):
            return [float(x) for x in s.split(",")]

        yaw = m.group(6).strip()
        cases.append({
            "origin": nums(m.group(1)), "dir": nums(m.group(2)), "normalize": bool(m.group(3)),
            "seed": int(m.group(4)), "preset": m.group(5),
            "light_yaw": "PI" if "PI" in yaw else float(yaw), "light_pitch": float(m.group(7)),
            "diamond_bits": [h(x) for x in re.findall(HEX, m.group(8))],
            "sapphire_bits": [h(x) for x in re.findall(HEX, sap)],
        })
    out["studio_cases"] = {"line": text[:start].count("\n") + 1, "max_bounces": 12, "cases": cases}

    # --- sample_studio_environment grid
    start = text.index("let env_expected: [[u32; 3]; 4] = [")
    body = start + len("let env_expected: [[u32; 3]; 4] = [")
    end = text.index("];\n", body)
    env = [[h(x) for x in re.findall(HEX, row)] for row in re.findall(r"\[([^\[\]]+)\]", text[body:end])]
    out["studio_env"] = {
        "line": text[:start].count("\n") + 1,
        "dirs_unnormalized": [[0.0, 1.0, 0.0], [0.5, 0.5, 0.5], [-0.3, 0.2, 0.9], [1.0, 0.0, 0.0]],
        "normalize": [False, True, True, False], "lambdas": [450.0, 550.0, 650.0],
        "preset": "RingLights", "exposure": 1.0, "light_yaw": 0.85, "light_pitch": 0.95, "bits": env,
    }

    # --- metrics
    start = text.index("let m = evaluate_gem_optical_metrics(&planes, &diamond, 0.0, 0.45, 0.85, 0.95);")
    end = text.index("],", text.index("],", start) + 2)
    vals = re.findall(HEX, text[start:end])
    out["metrics"] = {
        "line": text[:start].count("\n") + 1, "material": "Diamond", "cam_yaw": 0.0, "cam_pitch": 0.45,
        "light_yaw": 0.85, "light_pitch": 0.95,
        "fields": ["brilliance_pct", "fire_index", "scintillation_pct", "windowing_pct", "extinction_pct"],
        "bits": [h(v) for v in vals[:5]],
    }
    dst = Path(__file__).with_name("reference_goldens.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_goldens.py <gemray-studio checkout root>")
    main(sys.argv[1])
