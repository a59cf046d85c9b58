"""Extract the held-out split of a selector timing dataset into the fixture
``selector_heldout.npz`` used by tests/test_selector_cpu.py.

The dataset comes from timing every SpMM candidate plan on a B200 over the
seeded corpus (2000 training / 400 held-out matrices of at most 2^24
nonzeros, 40 held-out matrices above that, N in {1, 8, 32, 128}):

    python -m flagsparse_public_b200.tuning --train 2000 --test 400 --large 40 \\
        --steps 4000 --save-dataset sel_full.npz

which also trains and writes flagsparse_public_b200/selector_weights.npz.
Then:  python tests/golden/make_selector_fixture.py sel_full.npz
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(path):
    z = np.load(path, allow_pickle=False)
    test = ~z["split"].astype(bool)
    np.savez_compressed(os.path.join(HERE, "selector_heldout.npz"),
                        features=z["features"][test].astype(np.float64),
                        times=z["times"][test].astype(np.float32),
                        n_dense=z["n_dense"][test].astype(np.int16),
                        matrix=z["matrix"][test].astype(np.int32),
                        kind=z["kind"][test].astype(np.int8),
                        names=z["names"])


if __name__ == "__main__":
    main(sys.argv[1])
