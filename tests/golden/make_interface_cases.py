"""Extract the BM3D creation cases of the reference's interface golden.

Reads the reference's tests/data/plugin_interface_v1.json (recorded from the
CPU plugin by its tests/test_plugin_interface.py) and writes
bm3d_interface_cases.json beside this script: per case the clip format, the
keyword arguments of the call (decoded from the case key the way that test
builds it) and the expected outcome (output format/size or the exact error).
Run in a tree that has the reference checked out:

    python tests/golden/make_interface_cases.py --reference <reference checkout>

(or with the checkout's path in the NSS_REFERENCE environment variable).
"""
import argparse
import ast
import json
import os
from pathlib import Path

INT_PROBES = (-1, 0, 1, 2, 3, 4, 7, 8, 9, 16, 17, 33, 65, 1000)
FLOAT_PROBES = (-1.0, 0.0, 0.5, 1.0, 3.0, 1000.0)
INT_ARGS = {"block_size", "group_size", "block_step", "bm_range", "radius", "ps_num", "ps_range", "chroma", "final",
            "block_size_basic", "group_size_basic", "rolling_chunk", "rolling_cache_chunks", "rolling_cache_limit",
            "memory_limit_mb"}
FLOAT_ARGS = {"sigma", "sigma_basic"}


def decode(spec: str) -> dict:
    if spec == "defaults":
        return {}
    if spec.startswith("combo:"):
        body = spec[len("combo:"):]
        out = {}
        # keys are sorted, values are Python reprs; split on ",<name>=" boundaries
        parts, depth, cur = [], 0, ""
        for ch in body:
            if ch in "[(":
                depth += 1
            elif ch in "])":
                depth -= 1
            if ch == "," and depth == 0:
                parts.append(cur)
                cur = ""
            else:
                cur += ch
        parts.append(cur)
        for p in parts:
            k, v = p.split("=", 1)
            out[k] = ast.literal_eval(v)
        return out
    key, value = spec.split("=", 1)
    if value == "pair":
        probes = INT_PROBES if key in INT_ARGS else FLOAT_PROBES
        return {key: [probes[4], probes[3]]}
    return {key: ast.literal_eval(value)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("NSS_REFERENCE"))
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference checkout with --reference or NSS_REFERENCE")
    golden = json.loads((Path(args.reference) / "tests/data/plugin_interface_v1.json").read_text())
    cases = []
    for key in sorted(golden["cases"]):
        name, fmt, spec = key.split("|", 2)
        if name != "BM3D":
            continue
        cases.append({"key": key, "format": fmt, "kwargs": decode(spec), "expect": golden["cases"][key]})
    record = {
        "source": "reference tests/data/plugin_interface_v1.json (BM3D cases), recorded from the CPU plugin",
        "clip": {"width": 48, "height": 40, "frames": 4},
        "signature": golden["functions"]["BM3D"],
        "cases": cases,
    }
    out = Path(__file__).resolve().parent / "bm3d_interface_cases.json"
    out.write_text(json.dumps(record, indent=1, sort_keys=True) + "\n")
    print(f"wrote {out}: {len(cases)} cases")


if __name__ == "__main__":
    main()
