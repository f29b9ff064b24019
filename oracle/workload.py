"""Benchmark inputs for the reference CPU runs, written without this package's library (test
infrastructure: only tests, fixture generation and bench.py's reference / CPU-baseline legs use it).

* ``structured_msh``: the Gmsh 2.2 ASCII file of a structured mesh -- node lattice, boundary lines
  (bottom, right, top, left) with the physical tags of the boundary conditions, then the
  quadrilaterals row-major with their nodes in Gmsh order.  The reference reads it with
  simpleMesh::load (code/src/mesh/simpleMesh.cc:141-204).  Byte-for-byte the file that the
  library's ``dgb_mesh_write_msh`` writes (``tests/test_workload.py`` compares them).
* ``shock_bubble``: the seeded 2D shock-bubble initial state in the reference layout
  U[(e*N_F+f)*N_s+i] (gamma-model fields rho, rho u, rho v, E, 1/(gamma-1); the field
  definitions of init_cond.cc's multifluid initial conditions): a Mach-1.5 shock in air
  (gamma 1.4, pre-shock rho 1, p 1) at x = 0.2 moving in +x into a circular bubble of radius 0.2
  at (0.5, 0.5), gamma 1.67, rho 0.138, in pressure equilibrium, the radius perturbed by
  sum_k a_k cos((k+2) th + ph_k) with seeded a_k, ph_k.  The seed drives a 64-bit Mersenne
  twister (the published MT19937-64 algorithm) and uniform doubles x / 2^64, so the state is the
  library's ``init_state("shock_bubble", seed)`` bit for bit (same test).
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

BC_TAG = {"periodic": 1, "transmissive": 2, "reflective": 3, "frozen": 4}
MSH_LIN = {1: 1, 2: 8, 3: 26, 4: 27}   # Gmsh element types LIN_2 .. LIN_5
MSH_QUA = {1: 3, 2: 10, 3: 36, 4: 37}  # QUA_4 .. QUA_25
MSH_PNT = 15


class MT19937_64:
    """The 64-bit Mersenne twister (Matsumoto & Nishimura, MT19937-64 reference parameters)."""

    N, M = 312, 156
    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.mt = [0] * self.N
        self.mt[0] = seed & self.MASK
        for i in range(1, self.N):
            prev = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) & self.MASK
        self.idx = self.N

    def _twist(self):
        upper, lower = 0xFFFFFFFF80000000, 0x7FFFFFFF
        mt = self.mt
        for i in range(self.N):
            x = (mt[i] & upper) | (mt[(i + 1) % self.N] & lower)
            xa = x >> 1
            if x & 1:
                xa ^= 0xB5026F5AA96619E9
            mt[i] = mt[(i + self.M) % self.N] ^ xa
        self.idx = 0

    def next_u64(self) -> int:
        if self.idx >= self.N:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self.MASK

    def uniform01(self) -> float:
        """x / 2^64 rounded to a double, kept below 1 (a uniform double in [0, 1))."""
        v = float(self.next_u64()) / 18446744073709551616.0
        return v if v < 1.0 else math.nextafter(1.0, 0.0)


def quad_nodes(order: int) -> list[tuple[float, float]]:
    """Reference coordinates of the Gmsh QUA nodes of `order`: corners counter-clockwise from
    (-1, -1), the edge nodes edge by edge, then the interior nodes (recursively, scaled)."""
    if order == 0:
        return [(0.0, 0.0)]
    pts = [(-1.0, -1.0), (1.0, -1.0), (1.0, 1.0), (-1.0, 1.0)]
    if order > 1:
        corners = list(pts)
        for a, b in ((0, 1), (1, 2), (2, 3), (3, 0)):
            for i in range(1, order):
                pts.append((corners[a][0] + i * (corners[b][0] - corners[a][0]) / order,
                            corners[a][1] + i * (corners[b][1] - corners[a][1]) / order))
        s = 1.0 - 2.0 / order
        pts += [(x * s, y * s) for x, y in quad_nodes(order - 2)]
    return pts


def _lattice(n: int, a: float, b: float) -> np.ndarray:
    v = a + (b - a) * np.arange(n, dtype=np.float64) / float(n - 1)
    v[-1] = b
    return v


def element_node_offsets(order: int) -> tuple[np.ndarray, np.ndarray]:
    """Lattice offsets (di, dj) of the element's nodes in Gmsh order."""
    loc = quad_nodes(order)
    di = np.array([int(round((x + 1.0) * order / 2.0)) for x, _ in loc])
    dj = np.array([int(round((y + 1.0) * order / 2.0)) for _, y in loc])
    return di, dj


def structured_msh(path: str | Path, dim: int, order: int, nx: int, ny: int = 1, x0: float = 0.0,
                   x1: float = 1.0, y0: float = 0.0, y1: float = 1.0, bc=("transmissive",) * 4) -> None:
    """Write the Gmsh 2.2 file of a structured mesh (see the module docstring)."""
    tags = [BC_TAG[b] if isinstance(b, str) else int(b) for b in bc]
    lines = []
    p = order
    if dim == 1:
        N = p * nx + 1
        x = _lattice(N, x0, x1)
        lines += ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(N)]
        lines += [f"{i + 1} {x[i]:.17g} {0.0:.17g} {0.0:.17g}" for i in range(N)]
        lines += ["$EndNodes", "$Elements", str(nx + 2)]
        lines.append(f"1 {MSH_PNT} 2 {tags[0]} {tags[0]} 1")
        lines.append(f"2 {MSH_PNT} 2 {tags[1]} {tags[1]} {N}")
        for e in range(nx):
            nodes = [p * e, p * e + p] + [p * e + k for k in range(1, p)]
            lines.append(f"{e + 3} {MSH_LIN[p]} 2 100 100 " + " ".join(str(n + 1) for n in nodes))
        lines.append("$EndElements")
    else:
        NX, NY = p * nx + 1, p * ny + 1
        xs, ys = _lattice(NX, x0, x1), _lattice(NY, y0, y1)
        lines += ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(NX * NY)]
        sx = [f"{v:.17g}" for v in xs]
        sy = [f"{v:.17g}" for v in ys]
        z = f"{0.0:.17g}"
        k = 1
        for j in range(NY):
            for i in range(NX):
                lines.append(f"{k} {sx[i]} {sy[j]} {z}")
                k += 1
        nb = 2 * nx + 2 * ny
        lines += ["$EndNodes", "$Elements", str(nb + nx * ny)]

        def nid(i, j):
            return j * NX + i + 1

        def lin(idx):  # ends first, then the interior nodes in order
            return [idx[0], idx[-1]] + idx[1:-1]

        eid = 1
        sides = ([(tags[0], [nid(p * i + k, 0) for k in range(p + 1)]) for i in range(nx)] +
                 [(tags[1], [nid(NX - 1, p * j + k) for k in range(p + 1)]) for j in range(ny)] +
                 [(tags[2], [nid(p * i + k, NY - 1) for k in range(p + 1)]) for i in range(nx)] +
                 [(tags[3], [nid(0, p * j + k) for k in range(p + 1)]) for j in range(ny)])
        for tag, idx in sides:
            lines.append(f"{eid} {MSH_LIN[p]} 2 {tag} {tag} " + " ".join(str(n) for n in lin(idx)))
            eid += 1
        di, dj = element_node_offsets(p)
        t = MSH_QUA[p]
        for j in range(ny):
            for i in range(nx):
                nodes = " ".join(str(nid(p * i + a, p * j + b)) for a, b in zip(di, dj))
                lines.append(f"{eid} {t} 2 100 100 {nodes}")
                eid += 1
        lines.append("$EndElements")
    Path(path).write_text("\n".join(lines) + "\n")


def node_coordinates(order: int, nx: int, ny: int, x0: float, x1: float, y0: float, y1: float):
    """(X, Y) of every element node, shape (N_E, N_s), elements row-major, nodes in Gmsh order."""
    p = order
    xs, ys = _lattice(p * nx + 1, x0, x1), _lattice(p * ny + 1, y0, y1)
    di, dj = element_node_offsets(p)
    ii = (p * np.arange(nx))[None, :, None] + di[None, None, :]
    jj = (p * np.arange(ny))[:, None, None] + dj[None, None, :]
    X = np.broadcast_to(xs[ii], (ny, nx, len(di))).reshape(nx * ny, len(di))
    Y = np.broadcast_to(ys[jj], (ny, nx, len(di))).reshape(nx * ny, len(di))
    return X, Y


def shock_bubble(order: int, nx: int, ny: int, x0: float = 0.0, x1: float = 2.0, y0: float = 0.0,
                 y1: float = 1.0, seed: int = 7, xs: float = 0.2) -> np.ndarray:
    """The seeded shock-bubble state (module docstring), reference layout, float64."""
    g, M, rho1, p1 = 1.4, 1.5, 1.0, 1.0
    a1 = math.sqrt(g * p1 / rho1)
    p2 = p1 * (1.0 + 2.0 * g / (g + 1.0) * (M * M - 1.0))
    rho2 = rho1 * (g + 1.0) * M * M / ((g - 1.0) * M * M + 2.0)
    us = M * a1
    u2 = us * (1.0 - rho1 / rho2)
    rng = MT19937_64(seed)
    amp, ph = [], []
    for _ in range(8):
        amp.append(0.01 * 0.2 * (2.0 * rng.uniform01() - 1.0) / 8.0 * 2.0)
        ph.append(2.0 * math.pi * rng.uniform01())
    X, Y = node_coordinates(order, nx, ny, x0, x1, y0, y1)
    dx, dy = X - 0.5, Y - 0.5
    d2 = dx * dx + dy * dy
    # inside-bubble test r^2 > dx^2 + dy^2 with r = 0.2 + sum_k a_k cos((k+2) th + ph_k): |r - 0.2|
    # stays below sum |a_k| <= 0.004, so only nodes in that annulus need the exact libm sums
    bound = sum(abs(a) for a in amp)
    inside = d2 < (0.2 - bound - 1e-9) ** 2
    band = ~inside & (d2 < (0.2 + bound + 1e-9) ** 2)
    for idx in zip(*np.nonzero(band)):
        ddx, ddy = float(dx[idx]), float(dy[idx])
        th = math.atan2(ddy, ddx)
        r = 0.2
        for k in range(8):
            r += amp[k] * math.cos((k + 2) * th + ph[k])
        inside[idx] = ddx * ddx + ddy * ddy < r * r
    shocked = X < xs
    bub = ~shocked & inside
    rho = np.where(shocked, rho2, np.where(bub, 0.138, rho1))
    vx = np.where(shocked, u2, 0.0)
    vy = np.zeros_like(rho)
    pr = np.where(shocked, p2, p1)
    gam = np.where(bub, 1.67, g)
    ne, ns = X.shape
    U = np.empty((ne, 5, ns))
    U[:, 0] = rho
    U[:, 1] = rho * vx
    U[:, 2] = rho * vy
    U[:, 3] = 1.0 / (gam - 1.0) * pr + 0.5 * rho * (vx * vx + vy * vy)
    U[:, 4] = 1.0 / (gam - 1.0)
    return U.reshape(-1)
