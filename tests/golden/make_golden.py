"""Generate tests/golden/cook_3d_goldens.json from the reference's own
integration-test goldens (tests/*.prm + tests/*.output of
davydden/large-strain-matrix-free).  Run once where the reference tree is
available, giving its root directory:

    python tests/golden/make_golden.py <reference-root>

The JSON it writes is committed so that the test-suite never reads the
reference at run time.

Only the numbers are extracted: mesh size, reference volume, Newton
iteration counts and the displacement printed at the output point, plus the
parameter values of the matching .prm file.
"""
import json
import os
import re
import sys

CASES = ["cook_3d_quad_mf", "cook_3d_lin_mf"]


def parse_prm(text):
    out = {}
    for line in text.splitlines():
        line = line.split("#", 1)[0].strip()
        m = re.match(r"set\s+(.+?)\s*=\s*(.*)$", line)
        if m:
            out[m.group(1).strip()] = m.group(2).strip()
    return out


def parse_output(text):
    res = {"steps": []}
    m = re.search(r"Reference volume:\s*(\S+)", text)
    res["volume"] = float(m.group(1))
    res["n_cells"] = int(re.search(r"Number of active cells:\s*(\d+)", text).group(1))
    res["n_dofs"] = int(re.search(r"Number of degrees of freedom:\s*(\d+)", text).group(1))
    for blk in re.finditer(r"Timestep (\d+) @ (\S+)s\s*\nConverged in (\d+) Newton iterations\s*\n"
                           r"Solution @ ([^\n]*)\n\s*displacement: ([^\n]*)", text):
        res["steps"].append({"step": int(blk.group(1)), "time": float(blk.group(2)),
                             "newton_iterations": int(blk.group(3)),
                             "point": [float(v) for v in blk.group(4).split()],
                             "displacement": [float(v) for v in blk.group(5).split()]})
    return res


def main(ref_root):
    data = {}
    for c in CASES:
        with open(os.path.join(ref_root, "tests", c + ".prm")) as f:
            prm = parse_prm(f.read())
        with open(os.path.join(ref_root, "tests", c + ".output")) as f:
            out = parse_output(f.read())
        data[c] = {"source": "tests/%s.prm + tests/%s.output" % (c, c), "prm": prm, "output": out}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "cook_3d_goldens.json"), "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference-root>")
    main(sys.argv[1])
