"""Seeded synthetic SPD test matrices on grid patterns.

Value recipe (shared by the tests and the benchmark): the strictly lower
entries, taken in compressed-column order (column-major, rows ascending), are
i.i.d. N(0, 1) from `numpy.random.default_rng(seed)`; each diagonal entry is
the sum of |off-diagonal| over its full symmetric row plus 1, so the matrix is
strictly diagonally dominant and hence positive definite.  All generators
return the lower triangle (diagonal included) as a `spmatrix`.
"""
import numpy as np

from .sparse import spmatrix

__all__ = ["grid2d", "grid3d", "grid2d_extra", "random_lower", "spd_from_lower_pattern", "uneven_batch_specs"]


def spd_from_lower_pattern(n, I, J, seed):
    """Lower-triangular SPD matrix on the strictly-lower pattern (I > J)."""
    I = np.asarray(I, dtype=np.int64)
    J = np.asarray(J, dtype=np.int64)
    key = J * n + I
    key = np.unique(key)
    I, J = key % n, key // n
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(I.size)
    d = np.ones(n)
    np.add.at(d, I, np.abs(v))
    np.add.at(d, J, np.abs(v))
    ar = np.arange(n, dtype=np.int64)
    return spmatrix(np.concatenate([v, d]), np.concatenate([I, ar]), np.concatenate([J, ar]), (n, n))


def grid2d(nx, ny=None, seed=0):
    """5-point Laplacian pattern on an nx x ny grid (node = x + nx*y)."""
    ny = nx if ny is None else ny
    idx = np.arange(nx * ny).reshape(ny, nx)
    I = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()])
    J = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel()])
    return spd_from_lower_pattern(nx * ny, I, J, seed)


def grid3d(nx, ny=None, nz=None, seed=0):
    """7-point pattern on an nx x ny x nz grid (node = x + nx*(y + ny*z))."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    I = np.concatenate([idx[:, :, 1:].ravel(), idx[:, 1:, :].ravel(), idx[1:, :, :].ravel()])
    J = np.concatenate([idx[:, :, :-1].ravel(), idx[:, :-1, :].ravel(), idx[:-1, :, :].ravel()])
    return spd_from_lower_pattern(nx * ny * nz, I, J, seed)


def grid2d_extra(side, seed=0, extra=2, radius=5):
    """5-point grid of side x side where every node also gets `extra` random
    neighbours among the nodes within Manhattan distance <= radius that are
    not already adjacent (seeded; the batched-factorisation workload)."""
    n = side * side
    idx = np.arange(n).reshape(side, side)
    I = [idx[:, 1:].ravel(), idx[1:, :].ravel()]
    J = [idx[:, :-1].ravel(), idx[:-1, :].ravel()]
    rng = np.random.default_rng(seed + 1_000_003)
    offs = [(dx, dy) for dx in range(-radius, radius + 1) for dy in range(-radius, radius + 1)
            if 2 <= abs(dx) + abs(dy) <= radius]
    offs = np.array(offs, dtype=np.int64)
    xs = np.arange(n) % side
    ys = np.arange(n) // side
    # every node draws `extra` distinct candidates uniformly: random keys on
    # its candidate offsets, invalid ones pushed last, the smallest keys win
    cx = xs[:, None] + offs[None, :, 0]
    cy = ys[:, None] + offs[None, :, 1]
    ok = (cx >= 0) & (cx < side) & (cy >= 0) & (cy < side)
    keys = np.where(ok, rng.random(ok.shape), 2.0)
    k = min(extra, offs.shape[0])
    pick = np.argpartition(keys, k - 1, axis=1)[:, :k] if k > 0 else np.zeros((n, 0), dtype=np.int64)
    rows = np.arange(n)[:, None]
    valid = ok[rows, pick]
    u = (cx[rows, pick] + side * cy[rows, pick])[valid]
    v = np.broadcast_to(rows, pick.shape)[valid]
    ei = np.maximum(u, v)
    ej = np.minimum(u, v)
    I.append(np.asarray(ei, dtype=np.int64))
    J.append(np.asarray(ej, dtype=np.int64))
    seed_vals = int(rng.integers(0, 2**31 - 1)) ^ seed
    return spd_from_lower_pattern(n, np.concatenate(I), np.concatenate(J), seed_vals)


def random_lower(n, density, seed=0, diag=None):
    """Random strictly-lower pattern with about density*n*n candidate entries
    (values by the shared recipe, or a constant diagonal when `diag` given)."""
    rng = np.random.default_rng(seed)
    m = int(round(density * n * n))
    lin = rng.choice(n * n, size=m, replace=False)
    I, J = lin % n, lin // n
    keep = I > J
    A = spd_from_lower_pattern(n, I[keep], J[keep], seed + 17)
    if diag is not None:
        d = A._I == A._J
        V = A._V.copy()
        V[d] = diag
        A = spmatrix(V, A._I, A._J, A.size)
    return A


def uneven_batch_specs(count=256, seed=2024, lo=20, hi=120):
    """(side, seed) of each matrix of the batched workload: `count` 2-D grids
    with sides drawn uniformly from lo..hi (numpy default_rng(seed)); matrix i
    is grid2d_extra(side_i, seed=1000 + i)."""
    sides = np.random.default_rng(seed).integers(lo, hi + 1, size=count)
    return [(int(sd), 1000 + i) for i, sd in enumerate(sides)]
