"""Extracts the per-step log lines of the reference's captured runs.

Reads examples/tutorials/output2.param (power-law n=3) and output3.param
(afterslip) from a RELAX checkout and writes reference_logs.json: for each
run, the first log lines "I Dt tm(ve) tm(pl) tm(as) t/tmax power C:E^i"
(format 1100/1101 of src/relax.f90:1100-1105, 3 significant figures).
Run once where the reference is mounted:

    python tests/golden/make_reference_logs.py /path/to/relax
"""
import json
import os
import re
import sys

LINE = re.compile(r"^(\d{3})[* ]\s*(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)/(\S+)\s+(\S+)\s+(\S+)\s*$")


def parse(path, nlines):
    out = []
    with open(path) as f:
        for line in f:
            m = LINE.match(line.rstrip("\n"))
            if not m:
                continue
            i = int(m.group(1))
            vals = [float(m.group(k)) for k in (2, 3, 4, 5, 6, 8, 9)]
            out.append([i] + vals)
            if len(out) >= nlines:
                break
    return out


def main(root):
    tut = os.path.join(root, "examples", "tutorials")
    data = {
        "source": "examples/tutorials/output{2,3}.param of geodynamics/relax",
        "columns": ["i", "dt", "tm_ve", "tm_pl", "tm_as", "t", "power", "cei"],
        "output2": parse(os.path.join(tut, "output2.param"), 6),
        "output3": parse(os.path.join(tut, "output3.param"), 6),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_logs.json")
    with open(dst, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
