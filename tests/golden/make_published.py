"""Extracts the reference's published known answers for the time step into published.json.

Run once where the reference sources are available (its path is the only argument); the tests
read only the committed JSON. Sources:
  * docs/report/index.html:59 (commands at Makefile:41-43): grid, fluid nodes, threads and the
    FNV-1a state hash after `vortexlab bench --n 40 --steps 3000` and `--n 80 --steps 1000`;
  * README.md:182-188: the reference's own case-2D-2 results (c_D max / min, c_L max / min, St,
    pressure drop) at 20, 40 and 80 cells per diameter, lattice U = 0.05.
"""
import json
import os
import re
import sys


def hashes(root):
    line = open(os.path.join(root, "docs", "report", "index.html"), encoding="utf-8").read().splitlines()[58]
    out = {}
    for grid, nodes, threads, h in re.findall(
            r"<tr><td>(\d+x\d+)</td><td>(\d+)</td><td>(\d+)</td><td>\d+</td><td>[\d.]+x</td><td>([0-9a-f]{16})</td></tr>",
            line):
        steps = 3000 if grid == "882x166" else 1000
        n = 40 if grid == "882x166" else 80
        out.setdefault(grid, dict(n=n, steps=steps, fluid_nodes=int(nodes), hashes={}))["hashes"][threads] = h
    return out


def results_2d2(root):
    lines = open(os.path.join(root, "README.md"), encoding="utf-8").read().splitlines()[181:188]
    out = {}
    for line in lines:
        cells = [c.strip().replace("\u2212", "-") for c in line.strip().strip("|").split("|")]
        if len(cells) < 8 or cells[1] != "0.05" or not cells[0].isdigit() or "diverges" in cells[2]:
            continue
        nums = [float(re.findall(r"-?\d+\.\d+", c)[0]) for c in cells[2:8]]
        out[cells[0]] = dict(zip(("cd_max", "cd_min", "cl_max", "cl_min", "st", "dp"), nums))
    return out


if __name__ == "__main__":
    root = sys.argv[1]
    data = {"source": "useless-husband/vortexlab: docs/report/index.html:59, README.md:182-188",
            "bench_state_hashes": hashes(root), "case_2d2_u0.05": results_2d2(root)}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "published.json"), "w") as f:
        json.dump(data, f, indent=1)
        f.write("\n")
