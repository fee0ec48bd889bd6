"""Extract the reference's golden vectors into a small JSON fixture.

Reads ``benchmarks/tensorkit_semantic_oracle.out`` of the TeNeT checkout
(TensorKit main ``f87ca7f``, Julia 1.11.6, see that file's ``.jl`` header)
and writes ``tensorkit_semantic.json`` next to this script.  Run it only
where the reference checkout is present:

    python tests/golden/make_golden.py /root/reference

The committed JSON is what the tests read; the tests never read the
reference tree.
"""

import json
import re
import sys
from pathlib import Path


def parse(text):
    out = {
        "F_SU2": [],
        "R_SU2": [],
        "SU2_dim_twist_fs": [],
        "fZ2_twist_fs": [],
        "R_fZ2": [],
        "R_I3": [],
        "I3_twist_fs_dim": [],
        "streams": {},
        "repartition": [],
        "truncation": {},
    }
    section = None
    stream = None
    rep = None
    trunc = None
    for line in text.splitlines():
        m = re.match(r"== section (\d+)", line)
        if m:
            section = int(m.group(1))
            continue
        if section == 1:
            if m := re.match(r"F SU2 ((?:\d+ ){6})= (\S+)", line):
                out["F_SU2"].append([int(x) for x in m.group(1).split()] + [float(m.group(2))])
            elif m := re.match(r"R SU2 (\d+) (\d+) (\d+) = (\S+)", line):
                out["R_SU2"].append([int(m.group(i)) for i in (1, 2, 3)] + [float(m.group(4))])
            elif m := re.match(r"dim SU2 (\d+) = (\S+)\s+twist = (\S+)\s+fs = (\S+)", line):
                out["SU2_dim_twist_fs"].append([int(m.group(1))] + [float(m.group(i)) for i in (2, 3, 4)])
            elif m := re.match(r"twist fZ2 (\d) = (\S+)\s+fs = (\S+)", line):
                out["fZ2_twist_fs"].append([int(m.group(1)), float(m.group(2)), float(m.group(3))])
            elif m := re.match(r"R fZ2 (\d) (\d) = (\S+)", line):
                out["R_fZ2"].append([int(m.group(1)), int(m.group(2)), float(m.group(3))])
            elif m := re.match(r"R I3 \((\S+),(\S+),(\S+)\) \((\S+),(\S+),(\S+)\) -> \((\S+), (\S+), (\S+)\) = (\S+)", line):
                out["R_I3"].append([int(m.group(i)) for i in range(1, 10)] + [float(m.group(10))])
            elif m := re.match(r"twist I3 \((\S+),(\S+),(\S+)\) = (\S+)\s+fs = (\S+)\s+dim = (\S+)", line):
                out["I3_twist_fs_dim"].append([int(m.group(i)) for i in (1, 2, 3)] + [float(m.group(i)) for i in (4, 5, 6)])
        elif section == 3:
            if m := re.match(r"-- (\S+) --", line):
                stream = {"steps": {}, "svd": []}
                out["streams"][m.group(1)] = stream
            elif m := re.match(r"(s\d[ab]?) norm = (\S+)\s+tr = (\S+)", line):
                stream["steps"][m.group(1)] = [float(m.group(2)), float(m.group(3))]
            elif m := re.match(r"s6 svdcount = (\d+)", line):
                stream["svdcount"] = int(m.group(1))
            elif m := re.match(r"s6 svd\[(\d+)\] = (\S+)", line):
                stream["svd"].append(float(m.group(2)))
            elif m := re.match(r"s8 tr\(H\*H\) = (\S+)", line):
                stream["steps"]["s8"] = [float(m.group(1)), float(m.group(1))]
        elif section == 4:
            if m := re.match(r"-- (.+) --", line):
                rep = {"name": m.group(1)}
                out["repartition"].append(rep)
            elif m := re.match(r"ranks = (\d+),(\d+)", line):
                rep["ranks"] = [int(m.group(1)), int(m.group(2))]
            elif m := re.match(r"data = \[(.*)\]", line):
                rep["data"] = [float(x) for x in m.group(1).split(",")]
        elif section == 8:
            if m := re.match(r"-- (\S+) rank=(\d+) error=(\S+) --", line):
                trunc = {"rank": int(m.group(2)), "error": float(m.group(3)), "kept": []}
                out["truncation"][m.group(1)] = trunc
            elif m := re.match(r"sector (-?\d+) kept (\d+)", line):
                trunc["kept"].append([int(m.group(1)), int(m.group(2))])
    return out


def main():
    root = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
    src = root / "benchmarks" / "tensorkit_semantic_oracle.out"
    data = parse(src.read_text())
    data["source"] = "benchmarks/tensorkit_semantic_oracle.out (TensorKit main f87ca7f, Julia 1.11.6)"
    dst = Path(__file__).with_name("tensorkit_semantic.json")
    dst.write_text(json.dumps(data, indent=1))
    print(f"wrote {dst} ({dst.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
