"""Extract the reference's linear-solver test fixture into a JSON file.

Reads the 36x36 block system (12 blocks of 3x3, upper-triangular block
pattern), its right-hand side b, its solution x and its dense inverse from
g2o's unit_test/solver/sparse_system_helper.cpp and writes
tests/golden/sparse_system_36.json. The reference's own test
(unit_test/solver/linear_solver_test.cpp:84-101) solves this system twice and
requires isApprox(x, 1e-6).

Run once, in the container that holds the reference:
    python tests/golden/make_fixtures.py /path/to/g2o
"""
import json
import os
import re
import sys


def parse(src):
    text = open(src).read()

    def lines_of(fn):
        m = re.search(fn + r"\(\)\s*\{(.*?)\n\}", text, re.S)
        return m.group(1)

    body = lines_of(r"std::string sparseMatrixString")
    payload = " ".join(re.findall(r'aux << "([^"]*)"', body))
    tok = payload.split()
    pos = 0

    def take():
        nonlocal pos
        pos += 1
        return tok[pos - 1]

    assert take() == "RBI" and take() == ":"
    n = int(take())
    rbi = [int(take()) for _ in range(n)]
    assert take() == "CBI" and take() == ":"
    n = int(take())
    cbi = [int(take()) for _ in range(n)]
    blocks = []
    while pos < len(tok):
        assert take() == "BLOCK" and take() == ":"
        r, c = int(take()), int(take())
        rows = rbi[r] - (rbi[r - 1] if r else 0)
        cols = cbi[c] - (cbi[c - 1] if c else 0)
        vals = [float(take()) for _ in range(rows * cols)]
        blocks.append({"row": r, "col": c, "values": vals})
    inv_body = lines_of(r"std::string denseInverseMatrixString")
    inv_tok = " ".join(re.findall(r'aux << "([^"]*)"', inv_body)).split()
    assert inv_tok[:3] == ["#", "rows:", "36"], inv_tok[:6]
    inv = [float(v) for v in inv_tok[6:]]

    def vec(fn):
        return [float(v) for v in re.findall(r"result\(idx\+\+\) = ([-0-9.e+]+);", lines_of(fn))]

    b = vec(r"g2o::VectorX createTestVectorB")
    x = vec(r"g2o::VectorX createTestVectorX")
    return {"source": "unit_test/solver/sparse_system_helper.cpp", "row_block_indices": rbi,
            "col_block_indices": cbi, "blocks": blocks, "b": b, "x": x, "inverse": inv}


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <g2o source tree>")
    root = sys.argv[1]
    data = parse(os.path.join(root, "unit_test/solver/sparse_system_helper.cpp"))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sparse_system_36.json")
    with open(out, "w") as f:
        json.dump(data, f)
    print("wrote", out, len(data["blocks"]), "blocks", len(data["b"]), len(data["x"]), len(data["inverse"]))
