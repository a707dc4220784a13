"""Generate tests/golden/runtests_golden.json from MolecularIntegrals.jl's own test file.

The reference's known-answer values live in test/runtests.jl; this script reads that file
as text (nothing of the reference is executed) and writes the values, with the line each
came from, to a JSON fixture that the tests use.  Run where the reference is available:

    python tests/golden/make_golden.py <path to MolecularIntegrals.jl checkout>
"""
import json
import re
import sys
from pathlib import Path

NUM = r"[-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?)"


def testset(lines, title):
    start = next(i for i, ln in enumerate(lines) if f'@testset "{title}"' in ln)
    depth, out = 0, []
    for i in range(start, len(lines)):
        ln = lines[i]
        out.append((i + 1, ln))
        depth += len(re.findall(r"\b(?:begin|for|function|if)\b", ln))
        depth -= len(re.findall(r"^\s*end\b", ln))
        if i > start and depth == 0:
            break
    return out


def tuples(block, n):
    pat = re.compile(r"\(\s*" + r"\s*,\s*".join([f"({NUM})"] * n) + r"\s*\)")
    rows = []
    for lineno, ln in block:
        for m in pat.finditer(ln):
            rows.append({"line": lineno, "values": [float(x) for x in m.groups()]})
    return rows


def main():
    root = Path(sys.argv[1])
    path = root / "test" / "runtests.jl"
    lines = path.read_text().splitlines()
    gold = {"source": "MolecularIntegrals.jl test/runtests.jl"}

    vrr = testset(lines, "VRR tests")
    gold["vrr"] = [{"line": r["line"], "A": r["values"][0:3],
                    "a_ijk": [int(v) for v in r["values"][3:6]],
                    "c_ijk": [int(v) for v in r["values"][6:9]], "value": r["values"][9]}
                   for r in tuples(vrr, 10)]
    hrr = testset(lines, "HRR tests")
    gold["hrr"] = [{"line": r["line"], "A": r["values"][0:3],
                    "a_ijk": [int(v) for v in r["values"][3:6]], "b_ijk": [1, 0, 1],
                    "c_ijk": [int(v) for v in r["values"][6:9]], "d_ijk": [1, 0, 1],
                    "value": r["values"][9]} for r in tuples(hrr, 10)]

    one = testset(lines, "OneInts")
    fg = [ln for ln in one if "Fgamma" in ln[1] or "0.7468241328124271" in ln[1]]
    gold["fgamma"] = [{"line": r["line"], "m": int(r["values"][0]), "T": r["values"][1],
                       "value": r["values"][2]} for r in tuples(fg, 3)]

    eri = testset(lines, "ERI tests")
    sweep = [{"line": r["line"], "r": r["values"][0], "value": r["values"][1]}
             for r in tuples(eri, 2)]
    for lineno, ln in eri:  # (5.0, 1/5) style rows
        m = re.search(rf"\(\s*({NUM})\s*,\s*1/(\d+)\s*\)", ln)
        if m:
            sweep.append({"line": lineno, "r": float(m.group(1)), "value": 1.0 / int(m.group(2))})
    gold["ss_distance_sweep"] = sorted(sweep, key=lambda d: d["r"])
    named = {}
    for lineno, ln in eri:
        m = re.search(rf"@test coulomb\((.*)\)\s*(?:≈|==)\s*({NUM})\s*$", ln.strip())
        if m:
            named[m.group(1).replace(" ", "")] = {"line": lineno, "value": float(m.group(2))}
    gold["coulomb"] = named

    basis = testset(lines, "Basis")
    h2 = {}
    for lineno, ln in basis:
        m = re.search(rf"@test coulomb\(([lr]),([lr]),([lr]),([lr])\)\s*≈\s*({NUM})", ln)
        if m:
            h2["".join(m.groups()[:4])] = {"line": lineno, "value": float(m.group(5))}
    gold["h2_sto3g_coulomb"] = h2

    util = testset(lines, "Utils")
    ii = []
    for lineno, ln in util:
        if "iindex" not in ln:
            continue
        calls = re.findall(r"iindex\((\d+),(\d+),(\d+),(\d+)\)", ln)
        val = int(re.search(r"==\s*(\d+)\s*$", ln.strip()).group(1))
        for c in calls:
            ii.append({"line": lineno, "ijkl_1based": [int(x) for x in c], "value_1based": val})
    gold["iindex"] = ii

    dest = Path(__file__).with_name("runtests_golden.json")
    dest.write_text(json.dumps(gold, indent=1))
    print("wrote", dest, {k: len(v) for k, v in gold.items() if not isinstance(v, str)})


if __name__ == "__main__":
    main()
