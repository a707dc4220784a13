"""Extract the STO-3G table (H-Ne) of MolecularIntegrals.jl into sto3g.json.

STO-3G is published basis-set data (exponents and contraction coefficients); the engine
must use the exact numbers of the reference's table (src/Data.jl:5-120) for its results to
match the reference's, so they are read from that file rather than typed in.  Run once
where the reference source is available:

    python make_basis_data.py <path to MolecularIntegrals.jl checkout>
"""
import ast
import json
import sys
from pathlib import Path


def extract(src: str, name: str):
    start = src.index(f"\n{name} = [") + len(f"\n{name} = ")
    depth, i = 0, start
    while True:
        ch = src[i]
        if ch == "[":
            depth += 1
        elif ch == "]":
            depth -= 1
            if depth == 0:
                break
        i += 1
    body = "\n".join(line.split("#")[0] for line in src[start:i + 1].splitlines())
    return ast.literal_eval(body)


def main():
    root = Path(sys.argv[1])
    src = (root / "src" / "Data.jl").read_text()
    table = extract(src, "sto3g")
    out = {str(z + 1): [[sym, [[float(e), float(c)] for e, c in prims]] for sym, prims in shells]
           for z, shells in enumerate(table)}
    dest = Path(__file__).with_name("sto3g.json")
    dest.write_text(json.dumps({"source": "MolecularIntegrals.jl src/Data.jl:5-120 (sto3g)",
                                "elements": out}, indent=1))
    print("wrote", dest, len(out), "elements")


if __name__ == "__main__":
    main()
