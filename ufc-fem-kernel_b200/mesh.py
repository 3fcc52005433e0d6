"""Synthetic structured C3D8 meshes, Dirichlet sets and nodal loads.

The reference reads meshes through its L3 model-data layer (keyword parser);
this module stands in for it with seeded, structured boxes whose node and
element numbering follow the reference's conventions:

* node (i, j, k) has id ``i + (nx+1) * (j + (ny+1) * k)``;
* element (i, j, k) lists its nodes in Abaqus order, bottom face 1-4 then top
  face 5-8 (ufc_core/L4_PH/Element/PH_Elem_ShapeFunc.f90:329-350);
* DOF ``3 * node + comp`` (ufc_core/L5_RT/Assembly/RT_Asm_DofMap.f90:172-249).

Uniform tractions become consistent nodal forces through a 2x2 Gauss rule on
each loaded element face, as PH_Elem_C3D8_FormFacePressure does
(ufc_core/L4_PH/Element/Solid3D/PH_Elem_C3D8.f90:2360-2541).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MAT_ELASTIC_ISO = 101  # PH_Mat_Elas_Def.f90:24
MAT_J2_ISO = 201  # PH_Mat_Plast_Def.f90:17


@dataclass
class Problem:
    """A static C3D8 problem: mesh, material, Dirichlet set and load."""

    name: str
    shape: tuple  # (nx, ny, nz) elements
    coords: np.ndarray  # [N, 3] float64
    conn: np.ndarray  # [E, 8] int32, 0-based
    mat_model_id: int
    props: np.ndarray  # [E, nprops] float64: (E, nu) or (E, nu, sigma_y0, H)
    fixed: np.ndarray  # sorted unique int32 DOF ids
    fixed_values: np.ndarray  # float64, prescribed value per fixed DOF
    f: np.ndarray  # [3N] float64 external nodal forces (zero on fixed DOFs)
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.conn.shape[0])

    @property
    def n_dof(self) -> int:
        return 3 * self.n_nodes


def node_id(i, j, k, nx, ny):
    return i + (nx + 1) * (j + (ny + 1) * k)


def box_mesh(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float):
    """Structured hex mesh of the box [0,lx]x[0,ly]x[0,lz] with nx*ny*nz C3D8."""
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    zs = np.linspace(0.0, lz, nz + 1)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    coords = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1).astype(np.float64)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    n = lambda a, b, c: node_id(a, b, c, nx, ny)  # noqa: E731
    conn = np.stack(
        [n(i, j, k), n(i + 1, j, k), n(i + 1, j + 1, k), n(i, j + 1, k),
         n(i, j, k + 1), n(i + 1, j, k + 1), n(i + 1, j + 1, k + 1), n(i, j + 1, k + 1)],
        axis=1,
    ).astype(np.int32)
    return coords, conn


# Local node lists of the six hex faces, ordered so that the outward normal
# follows the right-hand rule (Abaqus face numbering S1..S6).
HEX_FACES = {
    "zmin": (0, 3, 2, 1), "zmax": (4, 5, 6, 7), "ymin": (0, 1, 5, 4),
    "xmax": (1, 2, 6, 5), "ymax": (2, 3, 7, 6), "xmin": (3, 0, 4, 7),
}


def face_traction(coords, conn, elems, face, traction, n_nodes=None):
    """Consistent nodal forces of a uniform traction vector on one face of the
    given elements, by a 2x2 Gauss rule on the bilinear face
    (PH_Elem_C3D8_FormFacePressure, PH_Elem_C3D8.f90:2360-2541)."""
    n_nodes = coords.shape[0] if n_nodes is None else n_nodes
    f = np.zeros(3 * n_nodes)
    loc = np.array(HEX_FACES[face])
    fn = conn[elems][:, loc]  # [F, 4]
    X = coords[fn]  # [F, 4, 3]
    g = 1.0 / np.sqrt(3.0)
    s4 = np.array([-1.0, 1.0, 1.0, -1.0])
    t4 = np.array([-1.0, -1.0, 1.0, 1.0])
    t = np.asarray(traction, dtype=np.float64)
    for s in (-g, g):
        for tt in (-g, g):
            N = 0.25 * (1 + s4 * s) * (1 + t4 * tt)
            dNs = 0.25 * s4 * (1 + t4 * tt)
            dNt = 0.25 * t4 * (1 + s4 * s)
            xs = np.einsum("a,fai->fi", dNs, X)
            xt = np.einsum("a,fai->fi", dNt, X)
            dA = np.linalg.norm(np.cross(xs, xt), axis=1)  # weight 1
            contrib = N[None, :, None] * dA[:, None, None] * t[None, None, :]
            for a in range(4):
                for c in range(3):
                    np.add.at(f, 3 * fn[:, a] + c, contrib[:, a, c])
    return f


def _face_elems(nx, ny, nz, face):
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    sel = {"xmax": i == nx - 1, "xmin": i == 0, "ymax": j == ny - 1, "ymin": j == 0,
           "zmax": k == nz - 1, "zmin": k == 0}[face]
    return np.nonzero(sel)[0]


def _plane_nodes(nx, ny, nz, axis, index):
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    c = (i, j, k)[axis].ravel()
    return np.nonzero(c == index)[0]


def _clamp(nodes):
    return np.sort(np.concatenate([3 * nodes, 3 * nodes + 1, 3 * nodes + 2])).astype(np.int32)


def cantilever(nx, ny, nz, lx, ly, lz, E=None, nu=0.3, traction=(0.0, 0.0, -1.0), name="cantilever"):
    """Clamped at x = 0 (all DOF), uniform traction on the x = lx face.
    E is a scalar or a per-element array."""
    coords, conn = box_mesh(nx, ny, nz, lx, ly, lz)
    ne = conn.shape[0]
    Ee = np.full(ne, 210e3) if E is None else np.broadcast_to(np.asarray(E, np.float64), (ne,)).copy()
    props = np.stack([Ee, np.full(ne, nu)], axis=1)
    fixed = _clamp(_plane_nodes(nx, ny, nz, 0, 0))
    f = face_traction(coords, conn, _face_elems(nx, ny, nz, "xmax"), "xmax", traction)
    f[fixed] = 0.0
    return Problem(name, (nx, ny, nz), coords, conn, MAT_ELASTIC_ISO, props, fixed,
                   np.zeros(fixed.size), f)


def lognormal_moduli(n_elems, seed, mu=np.log(210e3), sigma=0.5):
    return np.random.default_rng(seed).lognormal(mean=mu, sigma=sigma, size=n_elems)


def config1():
    """40x8x8 C3D8 cantilever on a 10x2x2 box, E = 210e3, nu = 0.3, clamped at
    x = 0, traction (0, 0, -1) on x = 10 (9,963 DOF)."""
    return cantilever(40, 8, 8, 10.0, 2.0, 2.0, E=210e3, name="cantilever_40x8x8")


def lognormal_cantilever(nx, ny, nz, seed, name=None):
    """Unit-spaced nx*ny*nz cantilever with per-element E ~ lognormal(ln 210e3, 0.5)."""
    ne = nx * ny * nz
    p = cantilever(nx, ny, nz, float(nx), float(ny), float(nz), E=lognormal_moduli(ne, seed),
                   name=name or f"lognormal_{nx}x{ny}x{nz}")
    p.meta["seed"] = seed
    return p


def config2():
    """128x64x64 unit-spaced cantilever, lognormal E (seed 2), 1,635,075 DOF."""
    return lognormal_cantilever(128, 64, 64, 2, "lognormal_128x64x64")


def config4():
    """192x96x96 unit-spaced cantilever, lognormal E (seed 4), 5,447,811 DOF."""
    return lognormal_cantilever(192, 96, 96, 4, "lognormal_192x96x96")


def j2_bar(nx=64, ny=32, nz=32, E=200e3, nu=0.3, sy=250.0, H=1000.0, name=None):
    """Displacement-controlled uniaxial J2 bar: u_x = 0 on x = 0, u_y = u_z = 0
    at node (0,0,0), u_z = 0 at node (0,ny,0); u_x on x = nx is prescribed per
    increment by :func:`j2_bar_target`."""
    coords, conn = box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    ne = conn.shape[0]
    props = np.tile(np.array([E, nu, sy, H]), (ne, 1))
    x0 = _plane_nodes(nx, ny, nz, 0, 0)
    x1 = _plane_nodes(nx, ny, nz, 0, nx)
    n000 = node_id(0, 0, 0, nx, ny)
    n0y0 = node_id(0, ny, 0, nx, ny)
    fixed = np.unique(np.concatenate([3 * x0, 3 * x1, [3 * n000 + 1, 3 * n000 + 2, 3 * n0y0 + 2]])).astype(np.int32)
    p = Problem(name or f"j2_bar_{nx}x{ny}x{nz}", (nx, ny, nz), coords, conn, MAT_J2_ISO, props, fixed,
                np.zeros(fixed.size), np.zeros(3 * coords.shape[0]))
    p.meta["pull_dofs"] = np.searchsorted(fixed, 3 * x1)
    p.meta["length"] = float(nx)
    return p


def j2_bar_target(p: Problem, step: int, n_steps: int = 20, strain: float = 0.01):
    """Prescribed values of the fixed DOFs at increment ``step`` (1-based):
    u_x = strain * L * step / n_steps on x = L, zero elsewhere."""
    v = np.zeros(p.fixed.size)
    v[p.meta["pull_dofs"]] = strain * p.meta["length"] * step / n_steps
    return v


def config3():
    """64x32x32 J2 bar, E = 200e3, nu = 0.3, sigma_y = 250, H = 1000."""
    return j2_bar(64, 32, 32, name="j2_bar_64x32x32")


def density_problem(nx, ny, nz, seed=5, n_rhs=16, name=None):
    """Per-element density rho ~ U(0.3, 1.0) (seed), E = 210e3 * rho^3, clamped
    at x = 0; n_rhs tip loads on the x = max face nodes
    f = (0, 0, -1) * (1 + 0.5 z), z ~ N(0, 1) per node, seed 50 + k."""
    coords, conn = box_mesh(nx, ny, nz, float(nx), float(ny), float(nz))
    ne = conn.shape[0]
    rho = np.random.default_rng(seed).uniform(0.3, 1.0, size=ne)
    props = np.stack([210e3 * rho ** 3, np.full(ne, 0.3)], axis=1)
    fixed = _clamp(_plane_nodes(nx, ny, nz, 0, 0))
    tip = _plane_nodes(nx, ny, nz, 0, nx)
    F = np.zeros((n_rhs, 3 * coords.shape[0]))
    for k in range(n_rhs):
        z = np.random.default_rng(50 + k).standard_normal(tip.size)
        F[k, 3 * tip + 2] = -(1.0 + 0.5 * z)
    p = Problem(name or f"density_{nx}x{ny}x{nz}", (nx, ny, nz), coords, conn, MAT_ELASTIC_ISO, props, fixed,
                np.zeros(fixed.size), F[0].copy())
    p.meta.update(rho=rho, F=F, tip_node=node_id(nx, ny // 2, nz // 2, nx, ny),
                  fd_elems=np.random.default_rng(seed).choice(ne, 32, replace=False))
    return p


def config5():
    """128x64x64 density problem, 16 tip-load right-hand sides."""
    return density_problem(128, 64, 64, 5, 16, "density_128x64x64")


def unit_cube_uniaxial(E=200e9, nu=0.3, sigma=100e6):
    """One C3D8 on the unit cube under uniaxial tension: x = 0 face fixed in x,
    node 1 fixed in y and z, node 4 in z, node 5 in y; 25e6 on each x-DOF of
    the x = 1 face (tests/ufc_core/test_c3d8_uniaxial.f90)."""
    coords, conn = box_mesh(1, 1, 1, 1.0, 1.0, 1.0)
    props = np.array([[E, nu]])
    # Abaqus nodes 1,4,5,8 are box nodes 0,2,4,6 (x = 0); 2,3,6,7 are 1,3,5,7.
    a = conn[0]
    fixed = np.array(sorted({3 * a[0], 3 * a[3], 3 * a[4], 3 * a[7], 3 * a[0] + 1, 3 * a[0] + 2,
                             3 * a[3] + 2, 3 * a[4] + 1}), dtype=np.int32)
    f = np.zeros(24)
    for nd in (a[1], a[2], a[5], a[6]):
        f[3 * nd] = sigma / 4.0
    return Problem("unit_cube_uniaxial", (1, 1, 1), coords, conn, MAT_ELASTIC_ISO, props, fixed,
                   np.zeros(fixed.size), f)


def free_mask(p: Problem):
    """Boolean mask of the free (not prescribed) DOFs."""
    m = np.ones(p.n_dof, dtype=bool)
    m[p.fixed] = False
    return m
