"""CPU oracle for the periodic homogenization solve (6 unit-strain load cases,
effective 6x6 elasticity tensor).

TEST INFRASTRUCTURE ONLY: the checker the CUDA homogenization path is
compared against; the product never imports it.

The reference has no counterpart: its "Homogenization" directory solves a
self-weight problem (Homogenization/QNC/QNC_V1_mod1m.m:180-199).  This file
restates the standard periodic homogenization of a voxel unit cell with the
same hex8 element matrix as the solver (oracle.hex8_stiffness, the
reference's Kem3 / Ke0):

  * nodes and elements on an n_x x n_y x n_z periodic grid share the index
    (n_z n_y) i + n_y k + j (y fastest, the reference's order); element
    (i, j, k) has the corners (i + x_a, j + y_a, k + z_a) mod n in the
    reference's local order x = {0,1,1,0,0,1,1,0}, y = {0,0,1,1,0,0,1,1},
    z = {0,0,0,0,1,1,1,1} (Cantilever/omp/mgcg1.c:621-624);
  * unit strain r (Voigt order xx, yy, zz, yz, xz, xy, engineering shears)
    has the affine field u0_r(x) = eps_r x; on an element it is u0_r at the
    corners' local coordinates (Ke annihilates translations, so the origin
    does not matter);
  * the periodic fluctuation chi_r solves K chi_r = -sum_e CX_e Ke u0_r,
    with node 0 held (it removes the rigid translations, the only null space
    of the periodic operator);
  * C_rs = (1 / n_el) sum_e CX_e (u0_r + chi_r)_e' Ke (u0_s + chi_s)_e.

Known answers used by the tests: a uniform cell gives C = CX D exactly (the
loads cancel at every node); a laminate of layers normal to x, one element or
more thick, gives the closed-form laminate tensor (the exact fluctuation is
piecewise linear in x, which the hex8 space holds); any cell lies between the
Reuss and Voigt bounds.
"""
from __future__ import annotations

import numpy as np

LX = np.array([0, 1, 1, 0, 0, 1, 1, 0])
LY = np.array([0, 0, 1, 1, 0, 0, 1, 1])
LZ = np.array([0, 0, 0, 0, 1, 1, 1, 1])


def node_index(i, j, k, nx, ny, nz):
    return (nz * ny) * (i % nx) + ny * (k % nz) + (j % ny)


def element_nodes(nx, ny, nz):
    """[nel, 8] node indices of every element (element order = node order)."""
    i, k, j = np.meshgrid(np.arange(nx), np.arange(nz), np.arange(ny), indexing="ij")
    i, k, j = i.reshape(-1), k.reshape(-1), j.reshape(-1)
    return np.stack([node_index(i + LX[a], j + LY[a], k + LZ[a], nx, ny, nz) for a in range(8)], axis=1)


def unit_strain_corners():
    """[6, 24]: u0_r at the eight local corners (x, y, z per corner)."""
    x, y, z = LX.astype(float), LY.astype(float), LZ.astype(float)
    zero = np.zeros(8)
    fields = [(x, zero, zero), (zero, y, zero), (zero, zero, z),
              (zero, z / 2, y / 2), (z / 2, zero, x / 2), (y / 2, x / 2, zero)]
    out = np.zeros((6, 24))
    for r, (ux, uy, uz) in enumerate(fields):
        out[r, 0::3], out[r, 1::3], out[r, 2::3] = ux, uy, uz
    return out


def isotropic_D(nu=0.3, E=1.0):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[[0, 1, 2], [0, 1, 2]] = lam + 2 * mu
    D[[3, 4, 5], [3, 4, 5]] = mu
    return D


def assemble(nx, ny, nz, CX, Ke):
    import scipy.sparse as sp
    en = element_nodes(nx, ny, nz)
    dof = (3 * en[:, :, None] + np.arange(3)[None, None, :]).reshape(len(en), 24)
    rows = np.repeat(dof, 24, axis=1).reshape(-1)
    cols = np.tile(dof, (1, 24)).reshape(-1)
    vals = (np.asarray(CX)[:, None] * Ke.reshape(1, -1)).reshape(-1)
    n = 3 * nx * ny * nz
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def loads(nx, ny, nz, CX, Ke):
    """[3N, 6]: the right-hand sides -sum_e CX_e Ke u0_r, assembled periodically."""
    en = element_nodes(nx, ny, nz)
    g = Ke @ unit_strain_corners().T            # [24, 6], the same for every element
    F = np.zeros((3 * nx * ny * nz, 6))
    for a in range(8):
        for d in range(3):
            np.add.at(F, 3 * en[:, a] + d, -np.asarray(CX)[:, None] * g[3 * a + d][None, :])
    return F


def homogenize(nx, ny, nz, CX, Ke):
    """(C_eff [6, 6], chi [3N, 6]) by a direct sparse solve with node 0 held."""
    import scipy.sparse.linalg as spl
    K = assemble(nx, ny, nz, CX, Ke)
    F = loads(nx, ny, nz, CX, Ke)
    n = K.shape[0]
    free = np.arange(3, n)
    chi = np.zeros((n, 6))
    Kf = K[free][:, free].tocsc()
    lu = spl.splu(Kf)
    chi[free] = lu.solve(F[free])
    return effective_tensor(nx, ny, nz, CX, Ke, chi), chi


def effective_tensor(nx, ny, nz, CX, Ke, chi):
    en = element_nodes(nx, ny, nz)
    dof = (3 * en[:, :, None] + np.arange(3)[None, None, :]).reshape(len(en), 24)
    u0 = unit_strain_corners()                  # [6, 24]
    W = u0[None, :, :] + np.transpose(chi[dof], (0, 2, 1))   # [nel, 6, 24]
    KW = np.einsum("ab,erb->era", Ke, W)
    C = np.einsum("e,era,esa->rs", np.asarray(CX), W, KW) / len(en)
    return C


def laminate(E_layers, frac, nu=0.3):
    """Effective tensor of isotropic layers normal to x (volume fractions
    frac, Young's moduli E_layers, common nu): the laminate formulas with the
    traction components N = (xx, xz, xy) continuous and the in-plane strains
    T = (yy, zz, yz) continuous across the layers."""
    N, T = [0, 4, 5], [1, 2, 3]
    Cs = [isotropic_D(nu, E) for E in E_layers]
    avg = lambda f: sum(w * f(C) for w, C in zip(frac, Cs))   # noqa: E731
    inv = np.linalg.inv
    A = inv(avg(lambda C: inv(C[np.ix_(N, N)])))
    B = avg(lambda C: inv(C[np.ix_(N, N)]) @ C[np.ix_(N, T)])
    Ceff = np.zeros((6, 6))
    Ceff[np.ix_(N, N)] = A
    Ceff[np.ix_(N, T)] = A @ B
    Ceff[np.ix_(T, N)] = (A @ B).T
    Ceff[np.ix_(T, T)] = avg(lambda C: C[np.ix_(T, T)] - C[np.ix_(T, N)] @ inv(C[np.ix_(N, N)]) @ C[np.ix_(N, T)]) \
        + B.T @ A @ B
    return Ceff


def voigt_reuss(CX, nu=0.3):
    """(Voigt, Reuss) bounds of an isotropic voxel cell with moduli CX."""
    D = isotropic_D(nu)
    return np.mean(CX) * D, D / np.mean(1.0 / np.asarray(CX))
