"""Write the Matrix Market test files under tests/golden/mtx/ and their CSR
golden outputs (tests/golden/mtx_golden.pt) produced by FlagSparse's own
loader, ``load_mtx_to_csr_torch`` (tests/test_spmv.py:103-178 of the
FlagSparse tree), run here with float64 values on the CPU.

The function is taken out of FlagSparse's test module by its source (the
module itself imports the GPU package at load time) and executed alone.

    python tests/golden/make_mtx_golden.py /path/to/FlagSparse
"""

import ast
import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
MTX_DIR = os.path.join(HERE, "mtx")

CASES = {
    "general_duplicates.mtx": """%%MatrixMarket matrix coordinate real general
% a comment line
%  another

5 4 9
1 1 1.5
2 3 -2.25
1 1 0.25
5 4 7e-3
6 1 9.0
3 0 1.0
2 3 2.25
4 2 0.0
1 4 -1e10
""",
    "symmetric.mtx": """%%MatrixMarket matrix coordinate real symmetric
4 4 6
1 1 4.0
2 1 1.0
3 1 -2.5
3 3 0.125
4 2 3.0
2 1 0.5
""",
    "skew.mtx": """%%MatrixMarket matrix coordinate real skew-symmetric
4 4 4
2 1 1.0
3 2 -0.75
4 1 2.0
4 3 5.5
""",
    "pattern_general.mtx": """%%MatrixMarket matrix coordinate pattern general
3 5 5
1 2
1 5
3 1
2 2
1 2
""",
    "pattern_symmetric.mtx": """%%MatrixMarket matrix coordinate pattern symmetric
4 4 4
1 1
3 1
4 2
4 4
""",
    "hermitian_complex.mtx": """%%MatrixMarket matrix coordinate complex hermitian
3 3 3
1 1 2.0 0.0
2 1 1.5 -0.5
3 2 -1.0 2.0
""",
    "integer_general.mtx": """%%MatrixMarket matrix coordinate integer general
3 3 4
1 1 3
2 2 -4
3 1 7
1 1 2
""",
    "short_header.mtx": """%%MatrixMarket matrix coordinate
2 2 2
1 2 1.0
2 1 -1.0
""",
    "array_format.mtx": """%%MatrixMarket matrix array real general
2 2
1.0
2.0
3.0
4.0
""",
    "empty.mtx": """%%MatrixMarket matrix coordinate real general
7 3 0
""",
    "crlf_upper.mtx": "%%MatrixMarket MATRIX Coordinate REAL Symmetric\r\n3 3 3\r\n1 1 1.0\r\n3 1 2.0\r\n2 2 -3.0\r\n",
}


def reference_loader(flagsparse_root):
    path = os.path.join(flagsparse_root, "tests", "test_spmv.py")
    tree = ast.parse(open(path).read())
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "load_mtx_to_csr_torch")
    ns = {"torch": torch}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), path, "exec"), ns)
    return ns["load_mtx_to_csr_torch"]


def main(flagsparse_root):
    os.makedirs(MTX_DIR, exist_ok=True)
    load = reference_loader(flagsparse_root)
    golden = {}
    for name, text in CASES.items():
        p = os.path.join(MTX_DIR, name)
        with open(p, "w", newline="") as fh:
            fh.write(text)
        data, indices, indptr, shape = load(p, dtype=torch.float64, device=torch.device("cpu"))
        golden[name] = {"data": data, "indices": indices, "indptr": indptr, "shape": torch.tensor(shape)}
    torch.save(golden, os.path.join(HERE, "mtx_golden.pt"))
    print(f"{len(golden)} cases")


if __name__ == "__main__":
    main(sys.argv[1])
