"""Pure-Python restatement of FlagSparse's Matrix Market loader.

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the native parser
(``fsb_mtx_open``) on files too large for the committed golden cases; the
library never imports it.  Follows load_mtx_to_csr_torch
(tests/test_spmv.py:103-178 of FlagSparse): per-row dicts summing in file
order from 0.0, mirrored symmetric / hermitian entries, negated
skew-symmetric mirrors, dropped out-of-range entries, sorted columns.
Pinned by tests/golden/mtx_golden.pt (FlagSparse's own outputs).
"""


def load(path):
    field, symmetry = "real", "general"
    header = None
    data_lines = []
    with open(path, "r", encoding="utf-8") as fh:
        for line in fh:
            s = line.strip()
            if s.startswith("%%MatrixMarket"):
                t = s.split()
                if len(t) >= 5:
                    field, symmetry = t[3].lower(), t[4].lower()
                continue
            if s.startswith("%"):
                continue
            if header is None and s:
                p = s.split()
                header = (int(p[0]), int(p[1]), int(p[2]) if len(p) > 2 else 0)
                continue
            if s:
                data_lines.append(s)
    n_rows, n_cols, nnz = header
    rows = [dict() for _ in range(n_rows)]
    if nnz:
        pattern = field == "pattern"
        sym = symmetry in ("symmetric", "hermitian")
        skew = symmetry == "skew-symmetric"
        for line in data_lines[:nnz]:
            p = line.split()
            r, c = int(p[0]) - 1, int(p[1]) - 1
            v = 1.0 if pattern else float(p[2])
            if 0 <= r < n_rows and 0 <= c < n_cols:
                rows[r][c] = rows[r].get(c, 0.0) + v
                if r != c and 0 <= c < n_rows and 0 <= r < n_cols:
                    if sym:
                        rows[c][r] = rows[c].get(r, 0.0) + v
                    elif skew:
                        rows[c][r] = rows[c].get(r, 0.0) - v
    indptr, indices, values = [0], [], []
    for row in rows:
        for c in sorted(row):
            indices.append(c)
            values.append(row[c])
        indptr.append(len(indices))
    return values, indices, indptr, (n_rows, n_cols)
