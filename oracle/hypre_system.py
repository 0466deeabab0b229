"""TEST INFRASTRUCTURE ONLY: the linear system of the reference's Hypre
pressure solver, assembled in numpy/scipy for checking the PCG + multigrid
solver of the CUDA library.

HyprePressureSolver::assembleSystem (src/HyprePressureSolver.cpp:154-279):
row i = (1 + c_i sum_f k_f) p_i - c_i sum_f k_f p_nb, c_i = rhoc2_i dt^2,
k_f = 1 / (max(rho_f, 1e-14) d_f w_i), rho_f the two-cell average, d_f the
mean of the two widths, w_i the cell's width along the face normal, k_f = 0
on non-periodic boundary faces.  Arrays are full (ghosted) context fields;
`geom` carries the extended cell widths (ghost widths included), the ghost
counts and the periodic flags."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def ext_widths(nodes, ng):
    """RectilinearMesh::buildExtendedNodes widths (src/RectilinearMesh.cpp:91-114):
    ghost widths mirror the first / last interior widths."""
    w = np.diff(np.asarray(nodes, dtype=np.float64))
    n = w.size
    lo = [w[min(g - 1, n - 1)] for g in range(ng, 0, -1)]
    hi = [w[max(n - g, 0)] for g in range(1, ng + 1)]
    return np.concatenate([lo, w, hi])


def assemble(dim, n, ng, widths, periodic, rho, rhoc2, rhs, dt):
    """(A, b) of the interior cells, x fastest; n = (nx, ny, nz), ng and
    widths per axis (widths include ghosts), periodic per axis."""
    nx, ny, nz = n
    gx, gy, gz = ng
    shape = (nz + 2 * gz, ny + 2 * gy, nx + 2 * gx)
    rho = rho.reshape(shape)
    rhoc2 = rhoc2.reshape(shape)
    rhs = rhs.reshape(shape)
    N = nx * ny * nz
    rows, cols, vals = [], [], []
    b = np.zeros(N)

    def lin(i, j, k):
        return (i % nx) + nx * ((j % ny) + ny * (k % nz))

    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                r = lin(i, j, k)
                idx = (k + gz, j + gy, i + gx)
                coeff = rhoc2[idx] * dt * dt
                diag = 0.0
                for ax in range(dim):
                    pos = (i, j, k)[ax]
                    nax = n[ax]
                    w = widths[ax]
                    g = ng[ax]
                    d = [0, 0, 0]
                    d[ax] = 1
                    for side in (-1, 1):
                        nb = (k + gz + side * d[2], j + gy + side * d[1], i + gx + side * d[0])
                        rf = 0.5 * (rho[idx] + rho[nb])
                        dd = 0.5 * (w[g + pos + side] + w[g + pos])
                        cc = 1.0 / (max(rf, 1e-14) * dd * w[g + pos])
                        if not periodic[ax] and ((side < 0 and pos == 0) or (side > 0 and pos == nax - 1)):
                            cc = 0.0
                        if cc != 0.0:
                            ii, jj, kk = i + side * d[0], j + side * d[1], k + side * d[2]
                            rows.append(r)
                            cols.append(lin(ii, jj, kk))
                            vals.append(-coeff * cc)
                        diag += cc
                rows.append(r)
                cols.append(r)
                vals.append(1.0 + coeff * diag)
                b[r] = rhs[idx]
    A = sp.csr_matrix((vals, (rows, cols)), shape=(N, N))
    return A, b


def solve(A, b):
    return spla.spsolve(A.tocsc(), b)
