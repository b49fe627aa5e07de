"""CPU FP64 restatement of the initial-field Poisson solve (test
infrastructure): the node charge density of the particles with the push's
rho shape (src/particle.cpp:503-514 weights, primal index (int)(x + 0.5)),
the 7-point Laplacian of the Yee grid with periodic or zero-flux axes, a
direct sparse solve, and E = -grad phi on the faces, in the reference
buffer layout."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def shape_weights(order: int, d: np.ndarray) -> np.ndarray:
    """B-spline weights (src/particle.cpp:8-48) for offsets d, shape (n, P)."""
    d = np.asarray(d, dtype=np.float64)
    if order == 2:
        return np.stack([0.5 * (0.5 - d) ** 2, 0.75 - d * d, 0.5 * (0.5 + d) ** 2], axis=1)
    a0, a1, a2, a3 = 55.0 / 96.0, 5.0 / 24.0, 5.0 / 4.0, 5.0 / 6.0
    b0, b2 = 115.0 / 192.0, 5.0 / 8.0
    u = d - 0.5
    w0 = u ** 4 / 24.0
    u = d + 1.0
    w1 = -u ** 4 / 6.0 + u ** 3 * a3 - u ** 2 * a2 + u * a1 + a0
    w2 = d ** 4 * 0.25 - d ** 2 * b2 + b0
    u = d - 1.0
    w3 = -u ** 4 / 6.0 - u ** 3 * a3 - u ** 2 * a2 - u * a1 + a0
    u = d + 0.5
    w4 = u ** 4 / 24.0
    return np.stack([w0, w1, w2, w3, w4], axis=1)


def node_rho(w, particles) -> np.ndarray:
    """Charge density of both species on the physical nodes, (nz, ny, nx)."""
    n = (w.nx, w.ny, w.nz)
    per = w.period
    order = 2 if w.mem == 2 else 4
    P = 3 if order == 2 else 5
    H = P // 2
    rho = np.zeros((w.nz, w.ny, w.nx))
    for kind, parts in enumerate(particles):
        if len(parts) == 0:
            continue
        q = w.species(kind)["charge"]
        pos = [np.array(parts[c], dtype=np.float64) for c in ("x", "y", "z")]
        idx, wts = [], []
        for d in range(3):
            v = pos[d].copy()
            if per[d]:
                v = np.where(v < 0.0, v + n[d], v)
                v = np.where(v > n[d], v - n[d], v)
            xc = v - (1 - w.mem)
            ip = (xc + 0.5).astype(np.int64)
            wts.append(shape_weights(order, xc - ip))
            idx.append(ip - H - w.mem)
        qw = q * np.asarray(parts["weight"], dtype=np.float64)
        for a in range(P):
            for b in range(P):
                for e in range(P):
                    val = qw * wts[2][:, a] * wts[1][:, b] * wts[0][:, e]
                    k, j, i = idx[2] + a, idx[1] + b, idx[0] + e
                    ok = np.ones(len(val), dtype=bool)
                    for c, m in ((i, 0), (j, 1), (k, 2)):
                        if per[m]:
                            c %= n[m]
                        else:
                            ok &= (c >= 0) & (c < n[m])
                    np.add.at(rho, (k[ok], j[ok], i[ok]), val[ok])
    return rho


def _lap1d(m: int, h: float, periodic: bool) -> sp.csr_matrix:
    """1D operator (2 phi_i - phi_{i+1} - phi_{i-1}) / h^2; zero flux at the
    ends of a non-periodic axis."""
    main = np.full(m, 2.0)
    off = -np.ones(m - 1)
    A = sp.diags([off, main, off], [-1, 0, 1], shape=(m, m), format="lil")
    if periodic:
        A[0, m - 1] -= 1.0
        A[m - 1, 0] -= 1.0
    else:
        A[0, 0] = 1.0
        A[m - 1, m - 1] = 1.0
    return (A.tocsr() / (h * h))


def solve_phi(w, rho: np.ndarray) -> tuple[np.ndarray, float]:
    """Mean-free solution of A phi = rho - <rho>; returns (phi, <rho>)."""
    mean = float(rho.mean())
    b = (rho - mean).ravel()
    nx, ny, nz = w.nx, w.ny, w.nz
    Ix, Iy, Iz = sp.identity(nx), sp.identity(ny), sp.identity(nz)
    Ax = _lap1d(nx, w.dx, bool(w.period[0]))
    Ay = _lap1d(ny, w.dy, bool(w.period[1]))
    Az = _lap1d(nz, w.dz, bool(w.period[2]))
    # x fastest: kron(z, y, x)
    A = sp.kron(Iz, sp.kron(Iy, Ax)) + sp.kron(Iz, sp.kron(Ay, Ix)) + sp.kron(Az, sp.kron(Iy, Ix))
    N = nx * ny * nz
    # the constants span the null space; adding the rank-one projector makes
    # the system regular and leaves the mean-free solution unchanged
    ones = np.ones(N) / np.sqrt(N)
    M = spla.LinearOperator((N, N), matvec=lambda v: A @ v + ones * (ones @ v), dtype=np.float64)
    phi, info = spla.cg(M, b, rtol=1e-14, atol=0.0, maxiter=20 * N)
    if info != 0:
        raise RuntimeError(f"reference CG did not converge ({info})")
    return phi.reshape(nz, ny, nx), mean


def fields_from_phi(w, phi: np.ndarray) -> dict:
    """E = -grad phi on the faces in the reference buffer layout; faces past
    the last node of a non-periodic axis are 0; periodic ghosts wrapped."""
    m = w.mem
    shape = (w.nz + 2 * m, w.ny + 2 * m, w.nx + 2 * m)
    out = {}
    for d, (name, h, axis) in enumerate((("ex", w.dx, 2), ("ey", w.dy, 1), ("ez", w.dz, 0))):
        nxt = np.roll(phi, -1, axis=axis)
        e = -(nxt - phi) / h
        if not w.period[d]:
            sl = [slice(None)] * 3
            sl[axis] = -1
            e[tuple(sl)] = 0.0
        buf = np.zeros(shape)
        buf[m:m + w.nz, m:m + w.ny, m:m + w.nx] = e
        for ax, pd in ((2, w.period[0]), (1, w.period[1]), (0, w.period[2])):
            if pd:
                nn = buf.shape[ax] - 2 * m
                lo = [slice(None)] * 3
                hi = [slice(None)] * 3
                src_lo = [slice(None)] * 3
                src_hi = [slice(None)] * 3
                lo[ax] = slice(0, m)
                src_lo[ax] = slice(nn, nn + m)
                hi[ax] = slice(m + nn, 2 * m + nn)
                src_hi[ax] = slice(m, 2 * m)
                buf[tuple(lo)] = buf[tuple(src_lo)]
                buf[tuple(hi)] = buf[tuple(src_hi)]
        out[name] = buf
    return out


def divergence(w, f: dict) -> np.ndarray:
    """(Ex(i+1/2) - Ex(i-1/2)) / dx + ... at the physical nodes."""
    m = w.mem
    z, y, x = slice(m, m + w.nz), slice(m, m + w.ny), slice(m, m + w.nx)
    ex, ey, ez = f["ex"], f["ey"], f["ez"]
    return ((ex[z, y, x] - ex[z, y, slice(m - 1, m - 1 + w.nx)]) / w.dx
            + (ey[z, y, x] - ey[z, slice(m - 1, m - 1 + w.ny), x]) / w.dy
            + (ez[z, y, x] - ez[slice(m - 1, m - 1 + w.nz), y, x]) / w.dz)
