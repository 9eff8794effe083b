"""Fit the polynomial of libisf's angle() kernel helper (isf_common.cuh).

atan(t) = t * P(t^2) on t in [0, 1]; P has degree DEG in s = t^2.  The fit
minimises the maximum absolute error of t*P(t^2) - atan(t) (Remez exchange
started from a Chebyshev-node least-squares fit), in double precision, then
rounds the coefficients to float32 and reports the error of a float32 Horner
evaluation.  Run:  python gen_atan_coeffs.py
"""
import numpy as np

DEG = 8


def design(t, deg):
    s = t * t
    return np.stack([t * s ** k for k in range(deg + 1)], axis=1)


def remez(deg, iters=30):
    n = deg + 2
    # Chebyshev extrema on [0, 1] as the initial reference
    t = 0.5 - 0.5 * np.cos(np.pi * np.arange(n) / (n - 1))
    grid = np.linspace(0, 1, 200001)
    for _ in range(iters):
        A = np.concatenate([design(t, deg), ((-1.0) ** np.arange(n))[:, None]], axis=1)
        sol = np.linalg.solve(A, np.arctan(t))
        c = sol[:-1]
        err = design(grid, deg) @ c - np.arctan(grid)
        # new reference: extrema of the error between sign changes
        idx = np.where(np.diff(np.sign(err)) != 0)[0]
        bounds = np.concatenate([[0], idx + 1, [len(grid)]])
        ext = [b0 + np.argmax(np.abs(err[b0:b1])) for b0, b1 in zip(bounds[:-1], bounds[1:]) if b1 > b0]
        if len(ext) < n:
            break
        ext = np.array(ext)
        # keep the n largest alternating extrema
        while len(ext) > n:
            k = np.argmin(np.abs(err[ext]))
            ext = np.delete(ext, k)
        t = grid[ext]
    return c


def f32_eval(c, t):
    c32 = c.astype(np.float32)
    t = t.astype(np.float32)
    s = t * t
    p = np.full_like(t, c32[-1])
    for k in range(len(c32) - 2, -1, -1):
        p = (p * s + c32[k]).astype(np.float32)
    return (t * p).astype(np.float32)


if __name__ == "__main__":
    c = remez(DEG)
    t = np.linspace(0, 1, 2000001)
    e64 = np.abs(design(t, DEG) @ c - np.arctan(t)).max()
    e32 = np.abs(f32_eval(c, t).astype(np.float64) - np.arctan(t)).max()
    print(f"degree {DEG}: minimax error {e64:.3e} (double), {e32:.3e} (float32 Horner)")
    for k, v in enumerate(c.astype(np.float32)):
        print(f"    c{k} = {float(v):.9e}f")
