"""FP64 oracle of the benchmark workload's log-determinant.

Builds the sparse SPD correlation matrix of bench.py (n = 262144 points
uniform in [0,1]^2 from numpy PCG64 seed 1, exp(-r/0.005) cut at 0.05,
diagonal shift 0.1) in float64 and computes logdet exactly from a sparse LU
factorisation (scipy.sparse.linalg.splu, MMD_AT_PLUS_A ordering, symmetric
mode): logdet = sum log|U_ii| (no negative pivots occur: the matrix is SPD).
Takes about five minutes on one core.

    python tests/golden/make_c2_oracle.py [n] [shift]
"""

import json
import os
import sys
import time

import numpy as np
import scipy.sparse.linalg as spl

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from imate_b200.sample_matrices import correlation_matrix  # noqa: E402


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 262144
    shift = float(sys.argv[2]) if len(sys.argv) > 2 else 0.1
    A = correlation_matrix(n, scale=0.005, threshold=0.05, shift=shift,
                           seed=1, dtype="float64", format="csc")
    t = time.time()
    lu = spl.splu(A, permc_spec="MMD_AT_PLUS_A",
                  options=dict(SymmetricMode=True))
    d = lu.U.diagonal()
    out = dict(n=n, shift=shift, nnz=int(A.nnz),
               logdet=float(np.sum(np.log(np.abs(d)))),
               negative_pivots=int(np.sum(d < 0)),
               method="splu MMD_AT_PLUS_A SymmetricMode, float64",
               seconds=round(time.time() - t, 1))
    with open(os.path.join(HERE, "c2prime_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
