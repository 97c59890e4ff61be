"""Extract the Float64x3 fused multiply-accumulate proof vectors from the
reference's test file into a JSON fixture.

Source: test/mulacc_x3_proof_vectors.jl:1-58 of MultiFloatLinearAlgebra.jl
(eight cases of UInt64 limb bit patterns for acc + x*y).  Run in a checkout
that has the reference mounted; the fixture it writes is committed so the
tests never read the reference at run time.

    python tests/golden/make_mulacc_x3_vectors.py /path/to/reference
"""
import json
import os
import re
import sys


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_mulacc_x3_vectors.py <reference checkout>")
    ref = sys.argv[1]
    src = os.path.join(ref, "test", "mulacc_x3_proof_vectors.jl")
    text = open(src).read()
    block = text[: text.index("@testset")]
    cases = []
    for m in re.finditer(r"name=:(\w+),(.*?)output=\(([^)]*)\)", block, re.S):
        name, body, out = m.group(1), m.group(2), m.group(3)
        fields = dict(re.findall(r"(acc|x|y)=\(([^)]*)\)", body))
        parse = lambda s: [v.strip() for v in s.split(",") if v.strip()]
        cases.append({
            "name": name,
            "acc": parse(fields["acc"]),
            "x": parse(fields["x"]),
            "y": parse(fields["y"]),
            "output": parse(out),
        })
    assert len(cases) == 8, len(cases)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mulacc_x3_proof_vectors.json")
    with open(dst, "w") as f:
        json.dump({"source": "test/mulacc_x3_proof_vectors.jl:1-58", "cases": cases}, f, indent=1)
    print("wrote", dst, len(cases), "cases")


if __name__ == "__main__":
    main()
