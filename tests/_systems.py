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


def isolated5(nx, ny, seed=0, dominance=1.05):
    """Vectorised 5-diagonal isolated system (plane-major S, W, P, E, N):
    off-diagonals U[-1, 0] on couplings between real cells, aP = 1.05
    sum|a_nb|, rhs N(0, 1) on real cells, zero-Dirichlet ghost ring."""
    rng = np.random.default_rng(seed)
    inner = np.zeros((ny, nx), bool)
    inner[1:-1, 1:-1] = True
    a = np.zeros((5, ny, nx))
    for k, (di, dj) in enumerate(OFF5):
        if k == 2:
            continue
        nb = np.zeros((ny, nx), bool)
        nb[max(0, -dj):ny - max(0, dj), max(0, -di):nx - max(0, di)] = \
            inner[max(0, dj):ny - max(0, -dj), max(0, di):nx - max(0, -di)]
        a[k] = np.where(inner & nb, -rng.uniform(0.0, 1.0, (ny, nx)), 0.0)
    a[2] = np.where(inner, dominance * np.abs(a).sum(axis=0), 1.0)
    b = np.where(inner, rng.standard_normal((ny, nx)), 0.0)
    return a.reshape(-1).copy(), b.reshape(-1).copy()
