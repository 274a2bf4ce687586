"""Extracts the golden data of the reference's captured runs.

Reads examples/tutorials/output2.param (power-law n = 3 after a strike-slip
fault), output3.param (afterslip on a frictional plane) and output4.param
(linear Maxwell with a weak zone and stress observation segments) from a
RELAX checkout and writes, next to this script:

* reference_logs.json -- for each run, every per-step log line
  "I Dt tm(ve) tm(pl) tm(as) t/tmax power C:E^i" (formats 1100/1101 of
  src/relax.f90:1100-1105, 3 significant figures);
* reference_outputN.input -- the input deck each log echoes
  (src/input.f90:43-1767 prints every record it reads, in reading order),
  turned back into an input file: numeric records are kept as they were
  printed, headers become comments, the output directory line keeps its
  name and the time line its skip and scaling.

output1.param is left out: it echoes an older form of the time line.

    python tests/golden/make_reference_logs.py <path to the RELAX checkout>
"""
import json
import os
import re
import sys

LINE = re.compile(r"^(\d{3})[* ]\s*(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)/(\S+)\s+(\S+)\s+(\S+)\s*$")
TIME = re.compile(r"^\s*(\S+)\s+\(output every (\d+) steps, dt scaled by (\S+)\)\s*$")
RUNS = ("output2", "output3", "output4")


def parse_log(path):
    out = []
    with open(path) as f:
        for line in f:
            m = LINE.match(line.rstrip("\n"))
            if not m:
                continue
            out.append([int(m.group(1))] + [float(m.group(k)) for k in (2, 3, 4, 5, 6, 8, 9)])
    return out


def _numeric(tokens):
    try:
        for t in tokens:
            float(t)
    except ValueError:
        return False
    return bool(tokens)


def echo_to_deck(path):
    """The echoed input of a log file as an input deck."""
    lines = open(path).read().splitlines()
    start = next(k for k, l in enumerate(lines) if l.startswith("grid dimension"))
    deck = [f"# input deck echoed in {os.path.basename(path)}"]
    prev = ""
    for line in lines[start:]:
        if line.startswith("max sampling size"):
            break
        tokens = line.split()
        if prev.startswith("output directory"):
            deck.append(tokens[0])
        elif TIME.match(line):
            m = TIME.match(line)
            deck.append(f"{m.group(1)} -{int(m.group(2))} {m.group(3)}")
        elif _numeric(tokens):
            deck.append(" ".join(tokens))
        else:
            deck.append("# " + line.strip())
        prev = line
    return "\n".join(deck) + "\n"


def main(root):
    tut = os.path.join(root, "examples", "tutorials")
    here = os.path.dirname(os.path.abspath(__file__))
    data = {"source": "examples/tutorials/output{2,3,4}.param of geodynamics/relax",
            "columns": ["i", "dt", "tm_ve", "tm_pl", "tm_as", "t", "power", "cei"]}
    for run in RUNS:
        src = os.path.join(tut, run + ".param")
        data[run] = parse_log(src)
        with open(os.path.join(here, f"reference_{run}.input"), "w") as f:
            f.write(echo_to_deck(src))
    with open(os.path.join(here, "reference_logs.json"), "w") as f:
        json.dump(data, f, indent=0)
    print("wrote", here, {r: len(data[r]) for r in RUNS})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
