"""Seeded synthetic linear systems for the solver tests.

dirichlet_system follows the isolated-system workload: off-diagonal
coefficients i.i.d. U[-1, 0], a_P = 1.05 * sum|a_nb|, right-hand side
N(0, 1), a zero-Dirichlet ghost ring (ghost rows a_P = 1, b = 0) and no
coupling from an interior cell to a ghost (those coefficients dropped).
"""
import numpy as np

# (di, dj) of each diagonal, reference order
OFF9 = [(-1, -1), (0, -1), (1, -1), (-1, 0), (0, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]
OFF5 = [(0, -1), (-1, 0), (0, 0), (1, 0), (0, 1)]


def offsets(nd):
    return OFF9 if nd == 9 else OFF5


def dirichlet_system(nd, nx, ny, seed=0, dominance=1.05):
    rng = np.random.default_rng(seed)
    N = nx * ny
    off = offsets(nd)
    kp = off.index((0, 0))
    a = np.zeros((nd, N))
    b = np.zeros(N)
    for j in range(ny):
        for i in range(nx):
            n = j * nx + i
            if i in (0, nx - 1) or j in (0, ny - 1):
                a[kp, n] = 1.0
                continue
            s = 0.0
            for k, (di, dj) in enumerate(off):
                if k == kp:
                    continue
                ii, jj = i + di, j + dj
                if ii in (0, nx - 1) or jj in (0, ny - 1):
                    continue           # coupling to the Dirichlet ring dropped
                v = -rng.uniform(0.0, 1.0)
                a[k, n] = v
                s += abs(v)
            a[kp, n] = dominance * s if s > 0 else 1.0
            b[n] = rng.standard_normal()
    return a.reshape(-1).copy(), b


def dense_from_planes(a, nd, nx, ny):
    N = nx * ny
    a = a.reshape(nd, N)
    A = np.zeros((N, N))
    for j in range(ny):
        for i in range(nx):
            n = j * nx + i
            for k, (di, dj) in enumerate(offsets(nd)):
                ii, jj = i + di, j + dj
                if 0 <= ii < nx and 0 <= jj < ny:
                    A[n, jj * nx + ii] += a[k, n]
    return A


def random_dominant_planes(nd, nx, ny, seed=0):
    """Random 9/5-diagonal system that respects only the solver's
    precondition (no coupling outside the grid); ghost rows are generic."""
    rng = np.random.default_rng(seed)
    N = nx * ny
    off = offsets(nd)
    kp = off.index((0, 0))
    a = np.zeros((nd, N))
    for j in range(ny):
        for i in range(nx):
            n = j * nx + i
            s = 0.0
            for k, (di, dj) in enumerate(off):
                if k == kp:
                    continue
                if 0 <= i + di < nx and 0 <= j + dj < ny:
                    v = rng.uniform(-1.0, 0.3)
                    a[k, n] = v
                    s += abs(v)
            a[kp, n] = 1.2 * s + rng.uniform(0.1, 1.0)
    b = rng.standard_normal(N)
    return a.reshape(-1).copy(), b


def tdma_lines_system(n, nlines, seed=0, dominance=1.05):
    rng = np.random.default_rng(seed)
    aw = -rng.uniform(0, 1, (nlines, n))
    ae = -rng.uniform(0, 1, (nlines, n))
    aw[:, 0] = 0.0
    ae[:, -1] = 0.0
    ap = dominance * (np.abs(aw) + np.abs(ae))
    ap[ap == 0] = 1.0
    d = rng.standard_normal((nlines, n))
    return aw, ap, ae, d
