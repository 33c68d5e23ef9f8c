"""Size-independent checks used where the CPU oracle cannot finish at full
size.  Each is exact; randomised ones state their error probability."""
import numpy as np


def freivalds_gemm(p, A, B, C0, C, a, b, trials=2, seed=0):
    """C == a*A*B + b*C0 (mod p) via random projections x: C x = a A (B x) +
    b C0 x.  Exact int64 arithmetic for p < 2^16, Python integers otherwise.
    A wrong C passes with probability at most p^-trials."""
    rng = np.random.default_rng(seed)
    dt = np.int64 if p < 2 ** 16 else object
    A = A.astype(dt); B = B.astype(dt); C0 = C0.astype(dt); C = C.astype(dt)
    for _ in range(trials):
        x = rng.integers(0, p, size=B.shape[1]).astype(dt)
        bx = (B @ x) % p
        lhs = (C @ x) % p
        rhs = (a * ((A @ bx) % p) + b * ((C0 @ x) % p)) % p
        if not np.array_equal(lhs, rhs):
            return False
    return True
