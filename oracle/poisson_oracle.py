"""Oracle (test infrastructure only): the reference's Poisson solve restated.

PoissonSolver (poissonSolver.pyx:33-88) on the finite-integration grid of
grid.pyx: the system matrix S diag(eps) S^T on the nodes of fixed-free
potential (S: the transposed discrete derivatives along x and y, stacked;
eps: epsilon_0 times the dual-edge over primal-edge ratios), factored by
SuperLU with the reference's options, and the node field E = N diag(1/ds) S^T
phi (N: edge-to-node interpolation).  The matrix products are formed in the
same order as the reference's so that phi and E agree bit for bit (the
grid's arrays come from the golden fixtures, which the compiled reference
wrote).  Not used by the product.
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl

EPSILON_0 = 8.85418781762e-12  # constants.pyx:8


class PoissonOracle:
    def __init__(self, nx_ext, inside_points, dsi, dst, edge_to_node):
        """nx_ext: nodes per row of the extended grid; inside_points: u16 per
        node (1 = free potential); dsi, dst: the grid's 2*np edge arrays
        (getDsi, getDst); edge_to_node: the (2 np, 2 np) sparse interpolation
        (getEdgeToNode)."""
        n = len(inside_points)
        self.n = n
        self.free = np.flatnonzero(np.asarray(inside_points))
        # transposed backward differences: column j of each block has +1 on
        # node j and -1 on the node after it along x (j + 1) or y (j + nx)
        ones = np.ones(n)
        d_x = sp.diags([ones, -ones[1:]], [0, -1], shape=(n, n))
        d_y = sp.diags([ones, -ones[nx_ext:]], [0, -nx_ext], shape=(n, n))
        s_t = sp.hstack([d_x, d_y])
        # material: eps_0 * (1 / ds) * dual-edge area, the dual areas of the
        # two blocks swapped (x edges take the y-block's dst and vice versa)
        eps = EPSILON_0 * np.asarray(dsi) * np.roll(np.asarray(dst), n)
        a = s_t.dot(sp.diags(eps, 0).dot(s_t.transpose()))[:, self.free].tocsc()[self.free, :]
        self.lu = spl.splu(a, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.1)
        self.phi_to_e = edge_to_node.dot(sp.diags(np.asarray(dsi), 0, (2 * n, 2 * n)).dot(s_t.transpose()))

    def solve(self, q):
        """Charge per dual cell (n) -> (phi (n), E at the nodes (2n): [Ex | Ey])."""
        phi = np.zeros(self.n)
        phi[self.free] = self.lu.solve(np.asarray(q, np.float64).take(self.free))
        return phi, self.phi_to_e.dot(phi)


def from_golden(z):
    """A PoissonOracle from a grid_*.npz fixture (its stored grid arrays; the
    edge-to-node matrix in the reference's own CSC order)."""
    nx = int(z["params"][0]) + 2
    n = z["insidePoints"].shape[0]
    e2n = sp.csc_matrix((z["e2n_csc_data"], z["e2n_csc_indices"], z["e2n_csc_indptr"]), shape=(2 * n, 2 * n))
    return PoissonOracle(nx, z["insidePoints"], z["Dsi"], z["Dst"], e2n)
