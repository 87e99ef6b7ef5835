"""Settings of the golden estimator runs of the other matrix functions
(functions.npz): shared by the generator (make_golden.py) and the tests."""

# (name, func, coefficients, gram, parameters) on the small correlation
# matrix (n = 400, scale 0.1, threshold 0.05, shift 0.1, seed 11)
FUNC_CASES = [
    ("exp_neg", "exp", [-1.0], False, None),
    ("exp_gram", "exp", [0.25], True, None),
    ("linfrac", "linfrac", [1.0, 2.0, 1.0, 3.0], False, None),
    ("indicator", "indicator", [0.5, 1.5], False, None),
    ("indicator_gram", "indicator", [0.0, 2.0], True, None),
    ("gaussian", "gaussian", [1.0, 0.3], False, None),
    ("gaussian_affine", "gaussian", [0.8, 0.5], False, [0.0, 0.3]),
    ("smoothstep", "smoothstep", [2.0], False, None),
]
FUNC_SETTINGS = dict(min_num_samples=10, max_num_samples=40, error_rtol=1e-2,
                     lanczos_degree=20, orthogonalize=-1, seed=7)
