"""Second, independent CPU restatement (numpy, vectorised) of the element and
material arithmetic, used to cross-check the C oracle.  Test infrastructure only.

Element: ComputeShape_Hex8 / ComputeJacobian / ComputeStrainDisplacementMatrix
(ufc_core/L4_PH/Element/PH_Elem_ShapeFunc.f90:125-350) and PH_Elem_Core_Compute_Ke
(ufc_core/L4_PH/Element/PH_Elem_Core.f90:95-166), 2x2x2 Gauss rule of
PH_Elem_GaussInt.f90:125-143.
Material: J2 radial return with linear isotropic hardening, written in tensor
(3x3) form rather than Voigt form so that the Voigt bookkeeping of the C oracle
and the CUDA kernels is checked against an independent formulation.
"""
from __future__ import annotations

import numpy as np

SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)
G1 = 1.0 / np.sqrt(3.0)
GAUSS = np.array([[(-G1, G1)[(ip >> 0) & 1], (-G1, G1)[(ip >> 1) & 1], (-G1, G1)[(ip >> 2) & 1]]
                  for ip in range(8)])


def shape_grad(xi):
    """dN/dxi [8,3] at one parametric point."""
    f = 1.0 + SIGNS * xi[None, :]
    d = np.empty((8, 3))
    d[:, 0] = 0.125 * SIGNS[:, 0] * f[:, 1] * f[:, 2]
    d[:, 1] = 0.125 * SIGNS[:, 1] * f[:, 0] * f[:, 2]
    d[:, 2] = 0.125 * SIGNS[:, 2] * f[:, 0] * f[:, 1]
    return d


def bmat(dNx):
    B = np.zeros((6, 24))
    for a in range(8):
        x, y, z = dNx[a]
        c = 3 * a
        B[0, c] = x; B[3, c] = y; B[5, c] = z
        B[1, c + 1] = y; B[3, c + 1] = x; B[4, c + 1] = z
        B[2, c + 2] = z; B[4, c + 2] = y; B[5, c + 2] = x
    return B


def iso_D(E, nu):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[range(3), range(3)] = lam + 2 * mu
    D[range(3, 6), range(3, 6)] = mu
    return D


def ke(X, D):
    K = np.zeros((24, 24))
    for xi in GAUSS:
        dN = shape_grad(xi)
        J = dN.T @ X  # J_ij = sum_k dN_k/dxi_i x_kj
        det = np.linalg.det(J)
        dNx = (np.linalg.inv(J) @ dN.T).T
        B = bmat(dNx)
        K += det * B.T @ D @ B
    return K


def voigt_to_tensor_strain(e):
    return np.array([[e[0], e[3] / 2, e[5] / 2], [e[3] / 2, e[1], e[4] / 2], [e[5] / 2, e[4] / 2, e[2]]])


def tensor_to_voigt_stress(s):
    return np.array([s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[1, 2], s[2, 0]])


def j2_tensor(props, deps_voigt, sig_n_voigt, epeq_n):
    """Tensor-form radial return; returns (sigma Voigt, epeq)."""
    E, nu, sy0, H = props
    G = E / (2 * (1 + nu))
    K = E / (3 * (1 - 2 * nu))
    de = voigt_to_tensor_strain(np.asarray(deps_voigt, dtype=np.float64))
    s_n = np.array(sig_n_voigt, dtype=np.float64)
    Sn = np.array([[s_n[0], s_n[3], s_n[5]], [s_n[3], s_n[1], s_n[4]], [s_n[5], s_n[4], s_n[2]]])
    St = Sn + K * np.trace(de) * np.eye(3) + 2 * G * (de - np.trace(de) / 3 * np.eye(3))
    p = np.trace(St) / 3
    dev = St - p * np.eye(3)
    q = np.sqrt(1.5 * np.sum(dev * dev))
    f = q - (sy0 + H * epeq_n)
    if f <= 0:
        return tensor_to_voigt_stress(St), epeq_n
    dg = f / (3 * G + H)
    S = (1 - 3 * G * dg / q) * dev + p * np.eye(3)
    return tensor_to_voigt_stress(S), epeq_n + dg


# ---------------------------------------------------------------- loads and output
# Face numbering and 2x2 face rule of PH_Elem_C3D8_FormFacePressure
# (ufc_core/L4_PH/Element/Solid3D/PH_Elem_C3D8.f90:2360-2541): face id ->
# (fixed parametric direction, its value, in-plane directions u and v, face nodes).
FACES = {1: (2, -1.0, 0, 1, (0, 1, 2, 3)), 2: (2, 1.0, 0, 1, (4, 7, 6, 5)),
         3: (1, -1.0, 0, 2, (0, 1, 5, 4)), 4: (1, 1.0, 0, 2, (3, 2, 6, 7)),
         5: (0, -1.0, 1, 2, (0, 3, 7, 4)), 6: (0, 1.0, 1, 2, (1, 5, 6, 2))}


def shape_n(xi):
    """N [8] at one parametric point (ComputeShape_Hex8, factor 1/8)."""
    return 0.125 * np.prod(1.0 + SIGNS * np.asarray(xi)[None, :], axis=1)


def face_load(X, face_id, traction=None, pressure=0.0):
    """Nodal forces [8,3] of one face: sum over the 2x2 face points of
    N_a (t - p n_out) dA, n_out the outward unit normal, found here from the
    element centroid (independent of the kernels' orientation table)."""
    fixed, val, ud, vd, nodes = FACES[face_id]
    t = np.zeros(3) if traction is None else np.asarray(traction, dtype=np.float64)
    F = np.zeros((8, 3))
    centroid = X.mean(axis=0)
    for gu in (-G1, G1):
        for gv in (-G1, G1):
            xi = np.zeros(3)
            xi[fixed], xi[ud], xi[vd] = val, gu, gv
            N = shape_n(xi)
            dN = shape_grad(xi)
            du, dv = dN[:, ud] @ X, dN[:, vd] @ X
            n = np.cross(du, dv)
            dA = np.linalg.norm(n)
            if dA < 1e-15:
                continue
            n /= dA
            if np.dot(n, N @ X - centroid) < 0:  # make it point away from the element
                n = -n
            F += np.outer(N, t - pressure * n) * dA
    for a in range(8):
        if a not in nodes:
            assert np.allclose(F[a], 0.0)
    return F


def face_loads(coords, conn, elem, face, traction=None, pressure=None):
    f = np.zeros(3 * coords.shape[0])
    for k in range(len(elem)):
        e = int(elem[k])
        X = coords[conn[e]]
        Fe = face_load(X, int(face[k]), None if traction is None else traction[k],
                       0.0 if pressure is None else pressure[k])
        for a in range(8):
            f[3 * conn[e, a]:3 * conn[e, a] + 3] += Fe[a]
    return f


def extrap_matrix():
    """(A^T)^-1 with A[a, ip] = N_a(Gauss point ip): nodal values from the
    eight Gauss-point values (PH_Elem_C3D8_GetExtrapMat, PH_Elem_C3D8.f90:2782-2800),
    Gauss points in the xi-fastest order of GAUSS."""
    A = np.stack([shape_n(g) for g in GAUSS], axis=1)  # [8 nodes, 8 points]
    return np.linalg.inv(A.T)


def nodal_stress(n_nodes, conn, sig_gp):
    """Extrapolate [E,8,6] Gauss-point stress to the element nodes and average
    over the elements sharing each node; returns ([N,6], von Mises [N])."""
    Ex = extrap_matrix()
    per_node = np.einsum("ai,eic->eac", Ex, sig_gp)
    s = np.zeros((n_nodes, 6))
    cnt = np.zeros(n_nodes)
    np.add.at(s, conn.ravel(), per_node.reshape(-1, 6))
    np.add.at(cnt, conn.ravel(), 1.0)
    s /= np.maximum(cnt, 1.0)[:, None]
    p = s[:, :3].mean(axis=1)
    j2 = 0.5 * ((s[:, :3] - p[:, None]) ** 2).sum(axis=1) + (s[:, 3:] ** 2).sum(axis=1)
    return s, np.sqrt(3.0 * np.maximum(j2, 0.0))
