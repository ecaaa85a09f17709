"""Structured Q2 box meshes and seeded synthetic operator inputs.

The arrays use the reference's single-rank local layouts (pTatin3D DMDA with
3 interleaved velocity dofs and box stencil width 2):

* node id ``i + j*X + k*X*Y`` with ``X = 2*mx+1``, ``Y = 2*my+1``
  (src/ptatin3d_stokes.c:121-146, src/dmda_element_q2p1.c:395-455);
* ``coords[3*N]``, ``u[3*N]`` interleaved (x, y, z) per node;
* ``eta[27*nel]`` element-major, quadrature-point minor with qp index
  ``a*9 + b*3 + c`` (c along xi), i.e. the ``QPntVolCoefStokes.eta`` order
  of include/QPntVolCoefStokes_def.h:41-46 and src/ptatin3d_stokes.c:466-475;
* ``p[4*nel]`` four P1 dofs per element;
* ``mask[3*N]`` uint8, nonzero on Dirichlet dofs (the BCList of
  src/dmda_bcs.c, scale 1).

The workloads follow the box-mesh configurations this project benchmarks
(unit box; perturbed interior nodes; log-uniform, sinker, layered or
per-element viscosity; Dirichlet on x-faces, free slip on y/z faces).  All
generators are seeded (``numpy.random.default_rng``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

GAUSS_X = np.array([-np.sqrt(3.0 / 5.0), 0.0, np.sqrt(3.0 / 5.0)])
GAUSS_W = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])


@dataclass
class BoxMesh:
    """A structured Q2 box mesh with mx*my*mz elements."""

    mx: int
    my: int
    mz: int
    coords: np.ndarray  # (3*N,) float64

    @property
    def dims(self):
        return (self.mx, self.my, self.mz)

    @property
    def nx(self):
        return 2 * self.mx + 1

    @property
    def ny(self):
        return 2 * self.my + 1

    @property
    def nz(self):
        return 2 * self.mz + 1

    @property
    def nnodes(self):
        return self.nx * self.ny * self.nz

    @property
    def nel(self):
        return self.mx * self.my * self.mz

    @property
    def nvel(self):
        return 3 * self.nnodes

    @property
    def npres(self):
        return 4 * self.nel


def box_coords(mx, my, mz, perturb=0.0, seed=0, extent=(1.0, 1.0, 1.0)):
    """Node coordinates of a Q2 box; every node moved by U(-perturb*h, perturb*h)
    per axis except along the normal of a boundary face it lies on (h = the
    element size along that axis)."""
    nx, ny, nz = 2 * mx + 1, 2 * my + 1, 2 * mz + 1
    xs = np.linspace(0.0, extent[0], nx)
    ys = np.linspace(0.0, extent[1], ny)
    zs = np.linspace(0.0, extent[2], nz)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    c = np.stack([X, Y, Z], axis=-1)  # (nz, ny, nx, 3)
    if perturb > 0.0:
        rng = np.random.default_rng(seed)
        h = np.array([extent[0] / mx, extent[1] / my, extent[2] / mz])
        d = rng.uniform(-1.0, 1.0, size=c.shape) * (perturb * h)
        d[:, :, 0, 0] = 0.0
        d[:, :, -1, 0] = 0.0
        d[:, 0, :, 1] = 0.0
        d[:, -1, :, 1] = 0.0
        d[0, :, :, 2] = 0.0
        d[-1, :, :, 2] = 0.0
        c = c + d
    return np.ascontiguousarray(c.reshape(-1))


def make_mesh(mx, my, mz, perturb=0.0, seed=0, extent=(1.0, 1.0, 1.0)):
    return BoxMesh(mx, my, mz, box_coords(mx, my, mz, perturb, seed, extent))


def element_table(mx, my, mz):
    """(nel, 27) int64 node ids, element e = ei + ej*mx + ek*mx*my."""
    X, Y = 2 * mx + 1, 2 * my + 1
    ek, ej, ei = np.meshgrid(np.arange(mz), np.arange(my), np.arange(mx), indexing="ij")
    base = (2 * ei + 2 * ej * X + 2 * ek * X * Y).reshape(-1)
    a, b, c = np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing="ij")
    off = (c + b * X + a * X * Y).reshape(-1)
    return base[:, None] + off[None, :]


def _q2_1d(t):
    return np.array([0.5 * t * (t - 1.0), (1.0 + t) * (1.0 - t), 0.5 * (1.0 + t) * t])


def qp_basis():
    """(27 qp, 27 nodes) Q2 basis values at the 3x3x3 Gauss points."""
    b = np.stack([_q2_1d(t) for t in GAUSS_X])  # [q][n]
    N = np.einsum("ak,bj,ci->abckji", b, b, b).reshape(27, 27)
    return N


def qp_coords(mesh: BoxMesh, chunk=1 << 16):
    """Physical coordinates of the 27 quadrature points of every element,
    shape (nel, 27, 3)."""
    N = qp_basis()
    el = element_table(*mesh.dims)
    c = mesh.coords.reshape(-1, 3)
    out = np.empty((mesh.nel, 27, 3))
    for s in range(0, mesh.nel, chunk):
        g = c[el[s:s + chunk]]
        out[s:s + chunk] = (N @ g.transpose(1, 0, 2).reshape(27, -1)).reshape(27, -1, 3).transpose(1, 0, 2)
    return out


# ---------------------------------------------------------------------------
# viscosity fields (eta at the 27 quadrature points of every element)
# ---------------------------------------------------------------------------

def eta_loguniform_qp(mesh: BoxMesh, lo=-2.0, hi=2.0, seed=1):
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(lo, hi, size=27 * mesh.nel)


def _qp_coords_of(mesh: BoxMesh, elems, comp=None):
    """Physical coordinates of the quadrature points of the given elements,
    shape (E, 27, 3) (or (E, 27) for one component)."""
    N = qp_basis()
    X, Y = mesh.nx, mesh.ny
    ei = elems % mesh.mx
    ej = (elems // mesh.mx) % mesh.my
    ek = elems // (mesh.mx * mesh.my)
    base = 2 * ei + 2 * ej * X + 2 * ek * X * Y
    a, b, c = np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing="ij")
    nid = base[:, None] + (c + b * X + a * X * Y).reshape(-1)[None, :]
    cc = mesh.coords.reshape(-1, 3)
    if comp is not None:
        return (cc[nid, comp] @ N.T)
    g = cc[nid]
    return np.einsum("qn,enc->eqc", N, g)


def eta_spheres(mesh: BoxMesh, centres, radii, values, background=1.0, layers=None, chunk=1 << 18):
    """Background (or horizontal layers along y) plus spherical inclusions,
    evaluated at the physical quadrature points; later spheres win.  Each
    sphere is tested only on the elements inside its index box (the
    generators perturb nodes by less than one element)."""
    eta = np.full((mesh.nel, 27), background, dtype=np.float64)
    if layers is not None:
        # layers: list of (y_top, value) from the bottom up
        for s in range(0, mesh.nel, chunk):
            y = _qp_coords_of(mesh, np.arange(s, min(s + chunk, mesh.nel)), comp=1)
            e = eta[s:s + chunk]
            lo = -np.inf
            for top, val in layers:
                e[(y >= lo) & (y < top)] = val
                lo = top
    cmin = mesh.coords.reshape(-1, 3).min(0)
    cmax = mesh.coords.reshape(-1, 3).max(0)
    m = np.array(mesh.dims)
    h = (cmax - cmin) / m
    for cc, r, v in zip(np.asarray(centres, dtype=np.float64).reshape(-1, 3), radii, values):
        lo = np.maximum(np.floor((cc - r - cmin) / h).astype(int) - 1, 0)
        hi = np.minimum(np.ceil((cc + r - cmin) / h).astype(int) + 1, m)
        if np.any(hi <= lo):
            continue
        kk, jj, ii = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]),
                                 indexing="ij")
        elems = (ii + mesh.mx * (jj + mesh.my * kk)).reshape(-1)
        xq = _qp_coords_of(mesh, elems)
        d2 = ((xq - cc[None, None, :]) ** 2).sum(-1)
        sub = eta[elems]
        sub[d2 <= r * r] = v
        eta[elems] = sub
    return np.ascontiguousarray(eta.reshape(-1))


def eta_sinker(mesh: BoxMesh, n=16, radius=0.08, eta_sphere=1e4, seed=1):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, size=(n, 3))
    return eta_spheres(mesh, centres, [radius] * n, [eta_sphere] * n)


def eta_layered(mesh: BoxMesh, n=64, radius=0.05, seed=1):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, 1.0, size=(n, 3))
    vals = 10.0 ** rng.uniform(-3.0, 3.0, size=n)
    layers = [(1.0 / 3.0, 1e3), (2.0 / 3.0, 1.0), (np.inf, 1e-1)]
    return eta_spheres(mesh, centres, [radius] * n, vals, layers=layers)


def eta_per_element(mesh: BoxMesh, contrast, seed=1):
    rng = np.random.default_rng(seed)
    e = 10.0 ** rng.uniform(0.0, np.log10(contrast), size=mesh.nel)
    return np.ascontiguousarray(np.repeat(e, 27))


# ---------------------------------------------------------------------------
# boundary conditions and vectors
# ---------------------------------------------------------------------------

def bc_mask_freeslip(mx, my, mz):
    """Dirichlet on all three components on the x-faces; the normal component
    on the y- and z-faces (free slip)."""
    nx, ny, nz = 2 * mx + 1, 2 * my + 1, 2 * mz + 1
    m = np.zeros((nz, ny, nx, 3), dtype=np.uint8)
    m[:, :, 0, :] = 1
    m[:, :, -1, :] = 1
    m[:, 0, :, 1] = 1
    m[:, -1, :, 1] = 1
    m[0, :, :, 2] = 1
    m[-1, :, :, 2] = 1
    return np.ascontiguousarray(m.reshape(-1))


def uniform_vec(n, seed, lo=-1.0, hi=1.0):
    return np.random.default_rng(seed).uniform(lo, hi, size=n)


def reference_test_vector(mesh: BoxMesh):
    """f = X + Y + Z + component + 3 per dof (src/tests/test_stokes_operators.c:81)."""
    c = mesh.coords.reshape(-1, 3)
    s = c.sum(axis=1)
    return np.ascontiguousarray((s[:, None] + np.arange(3)[None, :] + 3.0).reshape(-1))


def markers(mesh: BoxMesh, per_element=8, seed=1, contrast=1e4, n_incl=6, radius=0.15):
    """Seeded material points: per_element markers per element at uniform
    local coordinates, their physical positions through the Q2 map, and
    viscosity 1 or `contrast` (inside n_incl spheres), density 1 + 0.1 eta^0.
    Returns (wil int32[n], xi[n,3], x[n,3], eta[n], rho[n]); markers are
    listed element by element in a seeded random order."""
    rng = np.random.default_rng(seed)
    nel = mesh.nel
    wil = np.repeat(np.arange(nel, dtype=np.int32), per_element)
    xi = rng.uniform(-1.0, 1.0, size=(wil.size, 3))
    perm = rng.permutation(wil.size)
    wil, xi = wil[perm], xi[perm]
    # Q2 basis at the markers, physical coordinates
    el = element_table(*mesh.dims)
    c = mesh.coords.reshape(-1, 3)
    Nx, Ny, Nz = (_q2_1d(xi[:, d]) for d in range(3))         # [3][n]
    N = np.einsum("an,bn,cn->nabc", Nz, Ny, Nx).reshape(-1, 27)  # node a*9+b*3+c
    x = np.einsum("nk,nkd->nd", N, c[el[wil]])
    centres = rng.uniform(0.0, 1.0, size=(n_incl, 3))
    inside = np.zeros(wil.size, dtype=bool)
    for cc in centres:
        inside |= ((x - cc) ** 2).sum(axis=1) < radius * radius
    eta = np.where(inside, contrast, 1.0)
    rho = 1.0 + 0.1 * inside
    return wil.astype(np.int32), xi, x, eta, rho


def problem(config: str, seed: int = 0):
    """Seeded inputs of a named box-mesh workload.

    Returns (mesh, eta, mask).  Names: ``c0`` 8^3 perturbed +-0.1h with
    log-uniform eta in [1e-2, 1e2]; ``c1`` 64^3 undeformed sinker (16 spheres,
    r 0.08, eta 1e4); ``c2`` 128^3 perturbed +-0.05h layered with 64
    inclusions (contrast 1e6); ``box:mx,my,mz`` a perturbed box with
    log-uniform eta; ``sinker:mx,my,mz`` and ``layered:mx,my,mz`` the c1 and
    c2 viscosity fields on a box of that size (perturbed +-0.05h).
    """
    if config == "c0":
        m = make_mesh(8, 8, 8, perturb=0.1, seed=seed)
        eta = eta_loguniform_qp(m, -2.0, 2.0, seed=seed + 1)
    elif config == "c1":
        m = make_mesh(64, 64, 64)
        eta = eta_sinker(m, seed=seed + 1)
    elif config == "c2":
        m = make_mesh(128, 128, 128, perturb=0.05, seed=seed)
        eta = eta_layered(m, seed=seed + 1)
    elif config.startswith("box:"):
        mx, my, mz = (int(v) for v in config[4:].split(","))
        m = make_mesh(mx, my, mz, perturb=0.1, seed=seed)
        eta = eta_loguniform_qp(m, -2.0, 2.0, seed=seed + 1)
    elif config.startswith(("sinker:", "layered:")):
        kind, dims = config.split(":")
        mx, my, mz = (int(v) for v in dims.split(","))
        m = make_mesh(mx, my, mz, perturb=0.05, seed=seed)
        eta = (eta_sinker if kind == "sinker" else eta_layered)(m, seed=seed + 1)
    else:
        raise ValueError(f"unknown workload {config!r}")
    return m, eta, bc_mask_freeslip(*m.dims)
