"""Seeded synthetic quad meshes and initial states for the benchmark configs.

Random numbers come from SplitMix64 (one portable generator shared with any
other implementation): draw k of seed s is the k-th output of the stream
starting at state s.  Jittered meshes draw two values per node in node-index
order (x then y), for every node; boundary nodes discard theirs.

Node numbering is row-major with x fastest, node(i, j) = j*(nx+1) + i;
element(i, j) = j*nx + i with vertices counter-clockwise
(bottom-left, bottom-right, top-right, top-left), as Zhijian's quad elements.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import _lib as L

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """The first n outputs of SplitMix64 from state ``seed`` (uint64 array)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, n: int) -> np.ndarray:
    """n doubles in [0, 1) from the top 53 bits of SplitMix64."""
    return (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


@dataclasses.dataclass
class QuadMesh:
    xy: np.ndarray            # [n_nodes, 2] float64
    conn: np.ndarray          # [n_elem, 4] int64, CCW
    bnd: np.ndarray           # [n_bnd, 3] int64 (v0, v1, tag)
    tag_names: dict           # tag -> boundary type name

    @property
    def n_elem(self) -> int:
        return int(self.conn.shape[0])

    def bc_specs(self):
        """(tag, zj_bc_type) pairs of this mesh's boundary groups."""
        return [(t, L.BC_TYPES[n]) for t, n in sorted(self.tag_names.items())]


@dataclasses.dataclass
class MixedMesh:
    """Straight-sided quads and triangles: element e has etype[e] (0 triangle,
    1 quadrilateral) and nodes conn[offsets[e]:offsets[e+1]], counter-clockwise."""
    xy: np.ndarray            # [n_nodes, 2]
    etype: np.ndarray         # [n_elem] int32
    offsets: np.ndarray       # [n_elem + 1] int64
    conn: np.ndarray          # flat int64
    bnd: np.ndarray           # [n_bnd, 3] (v0, v1, tag)
    tag_names: dict

    @property
    def n_elem(self) -> int:
        return int(self.etype.shape[0])

    def element(self, e: int) -> np.ndarray:
        return self.conn[self.offsets[e]:self.offsets[e + 1]]

    def bc_specs(self):
        return [(t, L.BC_TYPES[n]) for t, n in sorted(self.tag_names.items())]


def split_quads(mesh: QuadMesh, fraction: float, seed: int) -> MixedMesh:
    """Split a seeded fraction of a Q1 quad mesh's elements into two
    triangles along a random diagonal: per element, in element order, two
    SplitMix64 draws u, w of the seed: split if u < fraction, along the
    0-2 diagonal if w < 1/2, else along 1-3."""
    r = uniform01(seed, 2 * mesh.n_elem).reshape(mesh.n_elem, 2)
    et, conn, off = [], [], [0]
    for e, (v0, v1, v2, v3) in enumerate(mesh.conn[:, :4].tolist()):
        if r[e, 0] < fraction:
            tris = ((v0, v1, v2), (v0, v2, v3)) if r[e, 1] < 0.5 else ((v0, v1, v3), (v1, v2, v3))
            for t in tris:
                et.append(0); conn += list(t); off.append(len(conn))
        else:
            et.append(1); conn += [v0, v1, v2, v3]; off.append(len(conn))
    return MixedMesh(mesh.xy.copy(), np.array(et, np.int32), np.array(off, np.int64),
                     np.array(conn, np.int64), mesh.bnd.copy(), dict(mesh.tag_names))


def structured_quads(nx: int, ny: int, x0: float, x1: float, y0: float, y1: float,
                     jitter: float = 0.0, seed: int = 0,
                     side_tags=(1, 1, 1, 1), tag_names=None) -> QuadMesh:
    """nx*ny quads on [x0,x1]x[y0,y1]; interior nodes moved by
    U(-jitter*h, +jitter*h) per coordinate (h the local spacing).
    side_tags = (bottom, right, top, left)."""
    hx, hy = (x1 - x0) / nx, (y1 - y0) / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1))
    ii = ii.ravel(); jj = jj.ravel()
    x = x0 + ii * hx
    y = y0 + jj * hy
    x[ii == nx] = x1
    y[jj == ny] = y1
    if jitter > 0.0:
        r = uniform01(seed, 2 * (nx + 1) * (ny + 1)).reshape(-1, 2)
        interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)
        x = np.where(interior, x + (2.0 * r[:, 0] - 1.0) * jitter * hx, x)
        y = np.where(interior, y + (2.0 * r[:, 1] - 1.0) * jitter * hy, y)
    xy = np.stack([x, y], axis=1).astype(np.float64)
    ei, ej = np.meshgrid(np.arange(nx), np.arange(ny))
    ei = ei.ravel(); ej = ej.ravel()
    n0 = ej * (nx + 1) + ei
    conn = np.stack([n0, n0 + 1, n0 + nx + 2, n0 + nx + 1], axis=1).astype(np.int64)
    b = []
    for i in range(nx):
        b.append((i, i + 1, side_tags[0]))
    for j in range(ny):
        b.append((j * (nx + 1) + nx, (j + 1) * (nx + 1) + nx, side_tags[1]))
    for i in range(nx):
        b.append((ny * (nx + 1) + i + 1, ny * (nx + 1) + i, side_tags[2]))
    for j in range(ny):
        b.append(((j + 1) * (nx + 1), j * (nx + 1), side_tags[3]))
    bnd = np.asarray(b, dtype=np.int64)
    if tag_names is None:
        tag_names = {t: "farfield" for t in set(side_tags)}
    return QuadMesh(xy, conn, bnd, dict(tag_names))


# Node positions of the Q2 (9-node) and Q4 (25-node) quads on the element's
# (order+1)^2 lattice, in the shape-function order of basis.cpp:717-847
# (corners counter-clockwise from (-1,-1), then edge nodes, then interior).
_Q2_LATTICE = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
_Q4_XI = [0, 4, 4, 0, 1, 2, 3, 4, 4, 4, 3, 2, 1, 0, 0, 0, 1, 2, 3, 1, 2, 3, 1, 2, 3]
_Q4_ETA = [0, 0, 4, 4, 0, 0, 0, 1, 2, 3, 4, 4, 4, 3, 2, 1, 1, 1, 1, 2, 2, 2, 3, 3, 3]


def curved_quads(nx: int, ny: int, order: int, x0: float, x1: float, y0: float, y1: float,
                 amp: float = 0.03, side_tags=(1, 1, 1, 1), tag_names=None) -> QuadMesh:
    """nx*ny curved quads of geometric order 2 or 4 on [x0,x1]x[y0,y1]: every
    node of the (order*nx+1) x (order*ny+1) lattice, element corners, edge
    and interior nodes alike, is moved by the smooth map
      x += amp (x1-x0) sin(pi s) sin(2 pi t),  y += amp (y1-y0) sin(2 pi s) sin(pi t)
    (s, t the lattice coordinates scaled to [0, 1]), which vanishes on the
    boundary: the outer edges stay straight, every interior edge is curved.
    Boundary edges are listed by their corner nodes (the reference's face
    tags), side_tags = (bottom, right, top, left)."""
    if order not in (2, 4):
        raise ValueError("order must be 2 or 4")
    mx, my = order * nx, order * ny
    ii, jj = np.meshgrid(np.arange(mx + 1), np.arange(my + 1))
    ii = ii.ravel(); jj = jj.ravel()
    s_, t_ = ii / mx, jj / my
    x = x0 + s_ * (x1 - x0) + amp * (x1 - x0) * np.sin(np.pi * s_) * np.sin(2.0 * np.pi * t_)
    y = y0 + t_ * (y1 - y0) + amp * (y1 - y0) * np.sin(2.0 * np.pi * s_) * np.sin(np.pi * t_)
    x[ii == 0] = x0; x[ii == mx] = x1
    y[jj == 0] = y0; y[jj == my] = y1
    xy = np.stack([x, y], axis=1).astype(np.float64)
    node = lambda a, b: b * (mx + 1) + a
    lat = _Q2_LATTICE if order == 2 else list(zip(_Q4_XI, _Q4_ETA))
    conn = []
    for ej in range(ny):
        for ei in range(nx):
            conn.append([node(order * ei + a, order * ej + b) for a, b in lat])
    conn = np.asarray(conn, dtype=np.int64)
    b = []
    for i in range(nx):
        b.append((node(order * i, 0), node(order * (i + 1), 0), side_tags[0]))
    for j in range(ny):
        b.append((node(mx, order * j), node(mx, order * (j + 1)), side_tags[1]))
    for i in range(nx):
        b.append((node(order * (i + 1), my), node(order * i, my), side_tags[2]))
    for j in range(ny):
        b.append((node(0, order * (j + 1)), node(0, order * j), side_tags[3]))
    if tag_names is None:
        tag_names = {t: "farfield" for t in set(side_tags)}
    return QuadMesh(xy, conn, np.asarray(b, dtype=np.int64), dict(tag_names))


# ------------------------------------------------------------- the configs --

def vortex_mesh(n: int = 20) -> QuadMesh:
    """Uniform n x n Q1 quads on [-10,10]^2, all boundaries far-field."""
    return structured_quads(n, n, -10.0, 10.0, -10.0, 10.0, 0.0, 0,
                            (1, 1, 1, 1), {1: "farfield"})


def tgv_mesh(n: int = 256, seed: int = 1, jitter: float = 0.15) -> QuadMesh:
    """n x n Q1 quads on [0,pi]^2, interior nodes jittered, slip walls."""
    return structured_quads(n, n, 0.0, math.pi, 0.0, math.pi, jitter, seed,
                            (1, 1, 1, 1), {1: "slipwall"})


# Solver keywords of the shear-layer configuration (make_params): Navier-Stokes
# at Re 2000, Pr 0.72, HLLC, p = 1/(gamma M^2) with M = 0.3.  The far field is
# at rest (Mach keyword 0: u_inf = v_inf = 0), matching the zero mean velocity
# of the layer; a far field moving at M = 0.3 drives an inflow against the
# lower half of the layer and the corners with the slip walls diverge several
# times sooner.
SHEAR_LAYER_PARAMS = dict(gamma=1.4, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.0, riemann="HLLC",
                          compat=False, viscous=True, Re=2000.0, Pr=0.72,
                          bcs=[(1, "slipwall"), (2, "farfield")])


def shear_layer_mesh(n: int = 384, seed: int = 3, fraction: float = 0.3) -> MixedMesh:
    """n x n quads on [0,1]^2 with a seeded 30% split into triangles; slip
    walls at y = 0, 1 (tag 1), far field at x = 0, 1 (tag 2)."""
    q = structured_quads(n, n, 0.0, 1.0, 0.0, 1.0, 0.0, 0, (1, 2, 1, 2),
                         {1: "slipwall", 2: "farfield"})
    return split_quads(q, fraction, seed)


def shear_layer(xy: np.ndarray, gamma: float = 1.4, mach: float = 0.3, delta: float = 0.02) -> np.ndarray:
    """u = 0.5 tanh((y - 0.5)/delta), v = 0.01 sin(2 pi x), rho = 1,
    p = 1/(gamma M^2)."""
    x, y = xy[..., 0], xy[..., 1]
    u = 0.5 * np.tanh((y - 0.5) / delta)
    v = 0.01 * np.sin(2.0 * math.pi * x)
    return prim_to_cons(np.ones_like(x), u, v, np.full_like(x, 1.0 / (gamma * mach * mach)), gamma)


def isentropic_vortex(xy: np.ndarray, gamma: float = 1.4, beta: float = 5.0,
                      u_inf: float = 0.5, v_inf: float = 0.0,
                      rho_scale: float = 1.0, p_scale: float = 1.0) -> np.ndarray:
    """Shu/Yee isentropic vortex at the origin, conserved variables.  The
    scales give the dimensional twin: rho*rho_scale, p*p_scale, velocities
    *sqrt(p_scale/rho_scale)."""
    x, y = xy[..., 0], xy[..., 1]
    r2 = x * x + y * y
    f = beta / (2.0 * math.pi) * np.exp(0.5 * (1.0 - r2))
    u = u_inf - f * y
    v = v_inf + f * x
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * math.pi ** 2) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho ** gamma / gamma
    vs = math.sqrt(p_scale / rho_scale)
    return prim_to_cons(rho * rho_scale, u * vs, v * vs, p * p_scale, gamma)


def shu_vortex(xy: np.ndarray, gamma: float = 1.4, beta: float = 5.0, u_inf: float = 0.5,
               v_inf: float = 0.0) -> np.ndarray:
    """The isentropic vortex in the normalisation that makes it an exact Euler
    solution (rho_inf = p_inf = 1, T = p/rho, p = rho^gamma): it advects
    unchanged with (u_inf, v_inf).  (isentropic_vortex above follows the
    benchmark's stated normalisation, p_inf = 1/gamma, whose temperature
    perturbation is a factor gamma too large for exact radial balance.)"""
    x, y = xy[..., 0], xy[..., 1]
    r2 = x * x + y * y
    f = beta / (2.0 * math.pi) * np.exp(0.5 * (1.0 - r2))
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * math.pi ** 2) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    return prim_to_cons(rho, u_inf - f * y, v_inf + f * x, rho ** gamma, gamma)


def taylor_green(xy: np.ndarray, gamma: float = 1.4, mach: float = 0.3) -> np.ndarray:
    x, y = xy[..., 0], xy[..., 1]
    u = np.sin(x) * np.cos(y)
    v = -np.cos(x) * np.sin(y)
    rho = np.ones_like(x)
    p = 1.0 / (gamma * mach * mach) + rho / 4.0 * (np.cos(2 * x) + np.cos(2 * y))
    return prim_to_cons(rho, u, v, p, gamma)


def prim_to_cons(rho, u, v, p, gamma):
    U = np.empty(np.shape(rho) + (4,), dtype=np.float64)
    U[..., 0] = rho
    U[..., 1] = rho * u
    U[..., 2] = rho * v
    U[..., 3] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return U


def random_state(n_elem: int, n_sp: int, seed: int, gamma: float = 1.4,
                 rho0: float = 1.0, p0: float = 1.0, amp: float = 0.1) -> np.ndarray:
    """Seeded smooth-free random state around (rho0, 0, 0, p0): every value is
    perturbed independently, so traces and derivatives exercise every term."""
    r = uniform01(seed, n_elem * n_sp * 4).reshape(n_elem, n_sp, 4) * 2.0 - 1.0
    c = math.sqrt(gamma * p0 / rho0)
    rho = rho0 * (1.0 + amp * r[..., 0])
    u = 0.5 * c * r[..., 1]
    v = 0.5 * c * r[..., 2]
    p = p0 * (1.0 + amp * r[..., 3])
    return prim_to_cons(rho, u, v, p, gamma)
