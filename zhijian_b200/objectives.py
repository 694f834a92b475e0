"""Objectives of the discrete adjoint on straight-sided (Q1) quad meshes:
the domain integral of the kinetic energy, J = int 1/2 rho |u|^2 dOmega,
evaluated with the Gauss-Legendre solution-point weights times |J| of the
bilinear element map, and its gradient dJ/dU in the state layout
[E][n_sp][4]."""
from __future__ import annotations

import numpy as np

from .meshgen import QuadMesh


def quadrature_weights(mesh: QuadMesh, P: int) -> np.ndarray:
    """w_i w_j |det d(x,y)/d(xi,eta)| at the solution points, [E][n_sp]
    (n_sp index = j*(P+1) + i with i along xi, as the solver's layout)."""
    xg, wg = np.polynomial.legendre.leggauss(P + 1)
    xy = mesh.xy[mesh.conn[:, :4]]                   # [E][4][2], CCW from (-1,-1)
    xi, eta = np.meshgrid(xg, xg)                    # [j][i]
    xi, eta = xi.ravel(), eta.ravel()
    # bilinear shape-function derivatives at each point, [n_sp][4]
    dxi = 0.25 * np.stack([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)], axis=1)
    deta = 0.25 * np.stack([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)], axis=1)
    x_xi = np.einsum("sa,ea->es", dxi, xy[..., 0])
    y_xi = np.einsum("sa,ea->es", dxi, xy[..., 1])
    x_eta = np.einsum("sa,ea->es", deta, xy[..., 0])
    y_eta = np.einsum("sa,ea->es", deta, xy[..., 1])
    det = x_xi * y_eta - x_eta * y_xi
    w = np.outer(wg, wg).ravel()
    return w[None, :] * np.abs(det)


def kinetic_energy(U: np.ndarray, wq: np.ndarray):
    """(J, dJ/dU) for J = sum wq * (m^2 + n^2) / (2 rho)."""
    rho, m, n = U[..., 0], U[..., 1], U[..., 2]
    ke = 0.5 * (m * m + n * n) / rho
    J = float(np.sum(wq * ke))
    G = np.zeros_like(U)
    G[..., 0] = -wq * ke / rho
    G[..., 1] = wq * m / rho
    G[..., 2] = wq * n / rho
    return J, G
