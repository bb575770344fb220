"""numpy/scipy restatement of PyTO's hex8 structural-FEA path (test oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product package.

Every function cites the reference file:line whose algorithm it restates
(paths are relative to the PyTO project root).  The restatement is vectorised
(no per-element Python loops) but keeps the reference's arithmetic: the same
numbering, the same quadrature, the same solver recurrences and stopping
tests, and the same material/filter/OC formulas.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spl

__all__ = [
    "grid_mesh", "nodes_on_plane", "ke_hex8", "constitutive_matrix",
    "simp_scaling", "simp_sensitivity", "ramp_scaling", "ramp_sensitivity",
    "assemble_K", "jacobi_inverse", "impose_dirichlet_bc", "solve_fixed",
    "pcg_scipy", "deflation_groups", "deflation_groups_box", "deflation_W", "dpcg",
    "compliance_and_gradient", "postprocess", "pnorm_stress_and_sensitivity",
    "solution_dotproduct_and_gradient", "smoothing_filter",
    "volume_constraint", "oc_update", "elements_with_forces", "topopt_oc",
    "cantilever_bc", "matvec_free", "matvec_ebe",
    "ke_hex8_thermal", "assemble_K_thermal", "thermal_scaling", "thermal_sensitivity",
    "mirror_filter", "extrude_filter",
]


# --------------------------------------------------------------------------
# a1: grid numbering  (src/hex_mesher.py:72-169, :1080-1095, :732-760)
# --------------------------------------------------------------------------
def grid_mesh(nelx: int, nely: int, nelz: int, elem_size=(1.0, 1.0, 1.0)) -> dict:
    """Node/element numbering of ``HexMesher.grid_mesh`` (src/hex_mesher.py:72-169).

    Node id = ix + (nelx+1)*iy + (nelx+1)*(nely+1)*iz (loops :104-109); element
    corner order :120-124; 27-neighbour table with -1 outside :126-151; element
    centres = mean of the 8 corner coordinates :153-156; edof :1080-1095.
    """
    sx, sy, sz = nelx + 1, nely + 1, nelz + 1
    nn = sx * sy * sz
    ne = nelx * nely * nelz
    iz, iy, ix = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
    node_indices = np.stack([ix.ravel(), iy.ravel(), iz.ravel(), np.zeros(nn, int)], 1).astype(np.int32)
    node_xyz = np.zeros((nn, 3))
    for i in range(3):
        node_xyz[:, i] = 0.0 + elem_size[i] * node_indices[:, i]
    ez, ey, ex = np.meshgrid(np.arange(nelz), np.arange(nely), np.arange(nelx), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    n0 = ez * sx * sy + ey * sx + ex
    off = np.array([0, 1, 1 + sx, sx, sx * sy, 1 + sx * sy, 1 + sx + sx * sy, sx + sx * sy])
    elemArray = (n0[:, None] + off[None, :]).astype(np.int32)
    eid = np.arange(ne)
    nb = np.empty((ne, 27), dtype=np.int64)
    k = 0
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                nb[:, k] = eid + dz * nelx * nely + dy * nelx + dx
                k += 1
    nb[ez == 0, 0:9] = -1
    nb[ez == nelz - 1, 18:27] = -1
    nb[np.ix_(ey == 0, [0, 1, 2, 9, 10, 11, 18, 19, 20])] = -1
    nb[np.ix_(ey == nely - 1, [6, 7, 8, 15, 16, 17, 24, 25, 26])] = -1
    nb[np.ix_(ex == 0, [0, 3, 6, 9, 12, 15, 18, 21, 24])] = -1
    nb[np.ix_(ex == nelx - 1, [2, 5, 8, 11, 14, 17, 20, 23, 26])] = -1
    nb[nb > ne - 1] = ne - 1
    elem_centers = np.sum(node_xyz[elemArray], axis=1) / 8.0
    edof = (3 * elemArray[:, :, None].astype(np.int64) + np.arange(3)).reshape(ne, 24)
    return dict(nelx=nelx, nely=nely, nelz=nelz, elem_size=tuple(float(h) for h in elem_size),
                num_nodes=nn, num_elems=ne, node_indices=node_indices, node_xyz=node_xyz,
                elemArray=elemArray, elemNeighborsArray=nb.astype(np.int32),
                elem_centers=elem_centers, edof=edof)


def nodes_on_plane(mesh: dict, axis: int, min_limit: bool) -> np.ndarray:
    """``getNodesOnBoundingBoxPlane`` (src/hex_mesher.py:732-760)."""
    grid = (mesh["nelx"], mesh["nely"], mesh["nelz"])
    col = mesh["node_indices"][:, axis]
    return np.where(col == (0 if min_limit else grid[axis]))[0]


# --------------------------------------------------------------------------
# a3: element stiffness (src/hex_element_stiffness.py:9-30, :113-141, :221-286)
# --------------------------------------------------------------------------
def constitutive_matrix(E: float, nu: float) -> np.ndarray:
    """Isotropic D (src/hex_element_stiffness.py:221-228); shear rows xy, yz, xz."""
    return (E / ((1.0 + nu) * (1.0 - 2.0 * nu))) * np.array([
        [1.0 - nu, nu, nu, 0.0, 0.0, 0.0],
        [nu, 1.0 - nu, nu, 0.0, 0.0, 0.0],
        [nu, nu, 1.0 - nu, 0.0, 0.0, 0.0],
        [0.0, 0.0, 0.0, (1.0 - 2.0 * nu) / 2.0, 0.0, 0.0],
        [0.0, 0.0, 0.0, 0.0, (1.0 - 2.0 * nu) / 2.0, 0.0],
        [0.0, 0.0, 0.0, 0.0, 0.0, (1.0 - 2.0 * nu) / 2.0]])


def ke_hex8(E: float, nu: float, elem_size=(1.0, 1.0, 1.0)) -> np.ndarray:
    """24x24 Ke of a box hex8, 2x2x2 Gauss (src/hex_element_stiffness.py:232-286).

    Gauss points in (xi, eta, zeta) tensor order (:45-47); isoparametric
    gradients (:113-141); Jacobian = dN @ xyz (:144-180); B rows
    xx, yy, zz, xy, yz, xz (:273-283); Ke = sum B^T D B det(J) w.
    """
    dx, dy, dz = elem_size
    nodes = np.array([[0, dx, dx, 0, 0, dx, dx, 0],
                      [0, 0, dy, dy, 0, 0, dy, dy],
                      [0, 0, 0, 0, dz, dz, dz, dz]], dtype=float).T
    c = constitutive_matrix(E, nu)
    g = np.array([-0.5773502691896257, 0.5773502691896257])
    pts = np.array([[a, b, cc] for a in g for b in g for cc in g])
    wts = np.ones(8)
    xis = np.array([-1, 1, 1, -1, -1, 1, 1, -1.0])
    etas = np.array([-1, -1, 1, 1, -1, -1, 1, 1.0])
    zetas = np.array([-1, -1, -1, -1, 1, 1, 1, 1.0])
    ke = np.zeros((24, 24))
    for gp in range(8):
        xi, eta, zeta = pts[gp]
        dN = np.stack([0.125 * xis * (1 + eta * etas) * (1 + zeta * zetas),
                       0.125 * (1 + xi * xis) * etas * (1 + zeta * zetas),
                       0.125 * (1 + xi * xis) * (1 + eta * etas) * zetas], axis=1)  # (8,3)
        jac = np.zeros((3, 3))
        for j in range(3):
            jac[:, j] = np.ascontiguousarray(dN[:, j]) @ nodes
        jinv = np.linalg.inv(jac)
        grad = np.array([jinv @ dN[n] for n in range(8)])  # (8,3)
        b = np.zeros((6, 24))
        for l in range(8):
            b[0, 3 * l] = grad[l, 0]
            b[1, 3 * l + 1] = grad[l, 1]
            b[2, 3 * l + 2] = grad[l, 2]
            b[3, 3 * l] = grad[l, 1]
            b[3, 3 * l + 1] = grad[l, 0]
            b[4, 3 * l + 1] = grad[l, 2]
            b[4, 3 * l + 2] = grad[l, 1]
            b[5, 3 * l] = grad[l, 2]
            b[5, 3 * l + 2] = grad[l, 0]
        ke += b.T @ c @ b * np.linalg.det(jac) * wts[gp]
    return ke


def ke_hex8_thermal(k: float, elem_size=(1.0, 1.0, 1.0)) -> np.ndarray:
    """8x8 conduction Ke of a box hex8, 2x2x2 Gauss (src/hex_element_stiffness.py:340-385):
    Ke = sum_g k B^T B det(J) w with B the 3x8 physical shape-function gradients."""
    dx, dy, dz = elem_size
    nodes = np.array([[0, dx, dx, 0, 0, dx, dx, 0],
                      [0, 0, dy, dy, 0, 0, dy, dy],
                      [0, 0, 0, 0, dz, dz, dz, dz]], dtype=float).T
    g = np.array([-0.5773502691896257, 0.5773502691896257])
    xis = np.array([-1, 1, 1, -1, -1, 1, 1, -1.0])
    etas = np.array([-1, -1, 1, 1, -1, -1, 1, 1.0])
    zetas = np.array([-1, -1, -1, -1, 1, 1, 1, 1.0])
    ke = np.zeros((8, 8))
    for xi in g:
        for eta in g:
            for zeta in g:
                dN = np.stack([0.125 * xis * (1 + eta * etas) * (1 + zeta * zetas),
                               0.125 * (1 + xi * xis) * etas * (1 + zeta * zetas),
                               0.125 * (1 + xi * xis) * (1 + eta * etas) * zetas], axis=1)
                jac = dN.T @ nodes
                b = np.linalg.solve(jac, dN.T)  # (3, 8) physical gradients
                ke += k * b.T @ b * np.linalg.det(jac)
    return ke


def assemble_K_thermal(mesh: dict, s: np.ndarray, Ke8: np.ndarray) -> sp.csr_matrix:
    """COO assembly of sum_e s_e Ke on the node DOFs (edofMatThermal = elemArray;
    src/hex_thermal_fea.py:44-48, :98-112)."""
    ea = mesh["elemArray"].astype(np.int64)
    I = np.repeat(ea, 8, axis=1).ravel()
    J = np.tile(ea, (1, 8)).ravel()
    V = np.einsum("ij,e->eij", Ke8, s).ravel()
    n = mesh["num_nodes"]
    return sp.coo_matrix((V, (I, J)), shape=(n, n)).tocsr()


def thermal_scaling(x, penal=1.0, kvoid=1e-8):
    """SIMP conductivity ``Kvoid + x^p (1-Kvoid)`` (src/topopt_material_model.py:109-110)."""
    return kvoid + (x ** penal) * (1.0 - kvoid)


def thermal_sensitivity(x, penal=1.0, kvoid=1e-8):
    """``p x^(p-1) (1-Kvoid)`` (src/topopt_material_model.py:151-152)."""
    return penal * (x ** (penal - 1.0)) * (1.0 - kvoid)


# --------------------------------------------------------------------------
# a4: material interpolation (src/topopt_material_model.py:76-139)
# --------------------------------------------------------------------------
def simp_scaling(x, penal=3.0, emin=1e-8):
    """SIMP ``Emin + x^p (1-Emin)`` (src/topopt_material_model.py:88-89)."""
    return emin + (x ** penal) * (1.0 - emin)


def simp_sensitivity(x, penal=3.0, emin=1e-8):
    """SIMP derivative ``p x^(p-1) (1-Emin)`` (src/topopt_material_model.py:130-131)."""
    return penal * (x ** (penal - 1.0)) * (1.0 - emin)


def ramp_scaling(x, q=5.0, emin=1e-8):
    """RAMP (src/topopt_material_model.py:90-91)."""
    return emin + x * (1.0 - emin) / (1.0 + (1.0 - x) * q)


def ramp_sensitivity(x, q=5.0, emin=1e-8):
    """RAMP derivative (src/topopt_material_model.py:132-133)."""
    return ((1.0 - emin) / (1.0 + (1.0 - x) * q) ** 2) * (1.0 + q * (1.0 - x))


# --------------------------------------------------------------------------
# a5/a2/a6: assembly, Dirichlet elimination, Jacobi PCG
# --------------------------------------------------------------------------
def assemble_K(mesh: dict, s: np.ndarray, Ke: np.ndarray, active=None) -> sp.csr_matrix:
    """COO assembly of sum_e s_e Ke then CSR (src/hex_structural_fea.py:47-50, :87-102)."""
    edof = mesh["edof"]
    if active is not None:
        edof = edof[active]
        s = s[active]
    ndof = 3 * mesh["num_nodes"]
    I = np.repeat(edof, 24, axis=1).ravel()
    J = np.tile(edof, (1, 24)).ravel()
    V = np.einsum("ij,e->eij", Ke, s).ravel()
    return sp.coo_matrix((V, (I, J)), shape=(ndof, ndof)).tocsr()


def jacobi_inverse(A: sp.spmatrix, eps_tol: float = 1e-12) -> np.ndarray:
    """Inverse diagonal with |d|<eps -> 1 (src/linear_solvers.py:71-87)."""
    d = A.diagonal().copy()
    d[np.abs(d) < eps_tol] = 1.0
    return 1.0 / d


def impose_dirichlet_bc(A: sp.csr_matrix, b: np.ndarray, fixed: np.ndarray, g: np.ndarray):
    """Lift and slice (src/bound_cond.py:40-70)."""
    free = np.setdiff1d(np.arange(b.shape[0]), fixed)
    bm = b.copy()
    bm -= A[:, fixed] * g
    return A[free, :][:, free], bm[free], free


def pcg_scipy(A, b, Minv, rtol):
    """scipy ``cg`` with the Jacobi preconditioner (src/linear_solvers.py:164-168).

    scipy stops on ||r||_2 < rtol * ||b||_2.  Returns (x, iterations).
    """
    it = [0]

    def cb(_):
        it[0] += 1
    M = sp.diags(Minv)
    x, info = spl.cg(A, b, M=M, rtol=rtol, maxiter=100000, callback=cb)
    return x, it[0]


def solve_fixed(K: sp.csr_matrix, f: np.ndarray, fixed: np.ndarray, g=None, method="direct",
                rtol=1e-8, dsolver=None):
    """``linear_solvers.solve`` with elimination + scatter (src/linear_solvers.py:136-202)."""
    if g is None:
        g = np.zeros(len(fixed))
    A, b, free = impose_dirichlet_bc(K, f, fixed, g)
    info = {}
    if method == "direct":
        x = spl.splu(A.tocsc()).solve(b)
    elif method == "pcg":
        x, info["iters"] = pcg_scipy(A, b, jacobi_inverse(A), rtol)
    elif method == "dpcg":
        W = dsolver["W"][free, :]
        x, info["iters"] = dpcg(A, b, W, jacobi_inverse(A), rtol=rtol)
    else:
        raise ValueError("Unknown solver type")
    u = np.zeros(f.shape)
    u[fixed] = g
    u[free] = x
    return u, info


def matvec_free(mesh, s, Ke, u, fixed):
    """Reduced operator applied on the full vector: y = P K P u, P zeroes fixed DOFs."""
    K = assemble_K(mesh, s, Ke)
    v = u.copy()
    v[fixed] = 0.0
    y = K @ v
    y[fixed] = 0.0
    return y


def matvec_ebe(nel, s, Ke, u, fixed=None, chunk=1 << 20):
    """K(s) u without assembling K, for grids too large for a CSR on the host:
    y = sum_e s_e Ke u_e scattered to the element's 24 DOFs (the action of the
    matrix assembled at src/hex_structural_fea.py:87-102), element corners in the
    order of src/hex_mesher.py:120-124.  With ``fixed`` the reduced operator of
    src/bound_cond.py:40-70 is applied on full-length vectors (fixed DOFs of u
    read as 0, of y written as 0).  Elements are processed in z-slabs of about
    ``chunk`` elements, so memory stays a few times the vector size."""
    nx, ny, nz = (int(v) for v in nel)
    sx, sy = nx + 1, ny + 1
    U = np.array(u, dtype=np.float64, copy=True)
    if fixed is not None:
        U[np.asarray(fixed)] = 0.0
    U = U.reshape(nz + 1, sy, sx, 3)
    Y = np.zeros_like(U)
    S = np.asarray(s, dtype=np.float64).reshape(nz, ny, nx)
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    dz = max(1, chunk // max(1, nx * ny))
    for z0 in range(0, nz, dz):
        z1 = min(nz, z0 + dz)
        ue = np.concatenate([U[z0 + c[2]:z1 + c[2], c[1]:c[1] + ny, c[0]:c[0] + nx, :] for c in corners],
                            axis=-1).reshape(-1, 24)
        ye = (ue @ Ke.T) * S[z0:z1].reshape(-1, 1)
        ye = ye.reshape(z1 - z0, ny, nx, 24)
        for k, c in enumerate(corners):
            Y[z0 + c[2]:z1 + c[2], c[1]:c[1] + ny, c[0]:c[0] + nx, :] += ye[..., 3 * k:3 * k + 3]
    y = Y.reshape(-1)
    if fixed is not None:
        y[np.asarray(fixed)] = 0.0
    return y


# --------------------------------------------------------------------------
# a7: aggregation deflation (src/deflation.py:86-229, :386-457, :504-584)
# --------------------------------------------------------------------------
def deflation_groups(node_xyz: np.ndarray, n_groups_desired: int, min_nodes: int = 15):
    """Box partition + small-group merge of ``create_deflation_groups``
    (src/deflation.py:86-229).  Returns (node_group int32, count, centre)."""
    nn = node_xyz.shape[0]
    n_groups_desired = min(n_groups_desired, int(nn / (1 + min_nodes)))
    xyz = node_xyz
    mins = np.array([np.min(xyz[:, 0]), np.min(xyz[:, 1]), np.min(xyz[:, 2])])
    L = np.array([np.max(xyz[:, i]) - mins[i] for i in range(3)])
    temp = L[0] * L[1] * L[2]
    alpha = (n_groups_desired / temp) ** (1.0 / 3)
    nX = max(round(alpha * L[0]), 1)
    nY = max(round(alpha * L[1]), 1)
    nZ = max(round(alpha * L[2]), 1)
    ntent = nX * nY * nZ
    size = np.array([L[0] / nX, L[1] / nY, L[2] / nZ])
    rel = xyz - mins
    idx = np.floor(rel / size).astype(np.int32)
    idx = np.minimum(idx, np.array([nX - 1, nY - 1, nZ - 1]))
    grp = (idx[:, 0] + nX * idx[:, 1] + nX * nY * idx[:, 2]).astype(np.int32)
    count = np.bincount(grp, minlength=ntent)
    centre = np.zeros((ntent, 3))
    for i in range(3):
        np.add.at(centre[:, i], grp, xyz[:, i])
    for gi in range(ntent):
        if count[gi] > 0:
            for i in range(3):
                centre[gi, i] /= count[gi]
    mapping = np.zeros(ntent, dtype=np.int32)
    cur = 0
    for gi in range(ntent):
        if count[gi] < min_nodes:
            mapping[gi] = -1
        else:
            mapping[gi] = cur
            cur += 1
    ngroups = cur
    if np.any(mapping == -1):
        small = np.where((mapping == -1) & (count > 0))[0]
        valid = np.where(count >= min_nodes)[0]
        if len(small) > 0:
            d = np.linalg.norm(centre[small][:, None, :] - centre[valid][None, :, :], axis=2)
            closest = valid[np.argmin(d, axis=1)]
            mapping[small] = mapping[closest]
        ok = grp != -1
        grp[ok] = mapping[grp[ok]]
        count = np.bincount(grp[ok], minlength=ngroups)
        centre = np.zeros((ngroups, 3))
        for i in range(3):
            np.add.at(centre[:, i], grp[ok], xyz[ok, i])
        for gi in range(ngroups):
            for i in range(3):
                centre[gi, i] /= count[gi]
    return grp, count, centre


def deflation_groups_box(mesh: dict, agg=(4, 4, 4)):
    """Element-box aggregates: node (ix,iy,iz) -> box (ix//ax, iy//ay, iz//az), the
    last partial layer of nodes folded into the preceding box.  Not a reference
    routine: this is the 4x4x4-element aggregation that config 2 names; centre =
    mean node coordinate as in src/deflation.py:146-153."""
    ni = mesh["node_indices"]
    dims = (mesh["nelx"], mesh["nely"], mesh["nelz"])
    nb = [max(1, dims[d] // agg[d]) for d in range(3)]
    gidx = [np.minimum(ni[:, d] // agg[d], nb[d] - 1) for d in range(3)]
    grp = (gidx[0] + nb[0] * (gidx[1] + nb[1] * gidx[2])).astype(np.int32)
    ng = nb[0] * nb[1] * nb[2]
    count = np.bincount(grp, minlength=ng)
    centre = np.zeros((ng, 3))
    for i in range(3):
        np.add.at(centre[:, i], grp, mesh["node_xyz"][:, i])
    centre /= count[:, None]
    return grp, count, centre


def deflation_W(node_xyz: np.ndarray, grp: np.ndarray, centre: np.ndarray, ngroups: int,
                modes: int = 6) -> sp.csr_matrix:
    """Rigid-body deflation matrix (src/deflation.py:386-457).

    Columns 6g+{0,1,2} translations, 6g+3 rotation about x (0,-z,y),
    6g+4 about y (z,0,-x), 6g+5 about z (-y,x,0); rel = xyz - centre[g].
    ``modes=3`` keeps the translations only (packed as 3g+c).
    """
    nn = node_xyz.shape[0]
    rel = node_xyz - centre[grp]
    n = np.arange(nn)
    if modes == 3:
        rows = np.concatenate([3 * n, 3 * n + 1, 3 * n + 2])
        cols = np.concatenate([3 * grp, 3 * grp + 1, 3 * grp + 2])
        vals = np.ones(3 * nn)
        return sp.coo_matrix((vals, (rows, cols)), shape=(3 * nn, 3 * ngroups)).tocsr()
    iW = np.concatenate([3 * n, 3 * n, 3 * n, 3 * n + 1, 3 * n + 1, 3 * n + 1, 3 * n + 2, 3 * n + 2, 3 * n + 2])
    jW = np.concatenate([6 * grp, 6 * grp + 4, 6 * grp + 5, 6 * grp + 1, 6 * grp + 3, 6 * grp + 5,
                         6 * grp + 2, 6 * grp + 3, 6 * grp + 4])
    sW = np.concatenate([np.ones(nn), rel[:, 2], -rel[:, 1], np.ones(nn), -rel[:, 2], rel[:, 0],
                         np.ones(nn), rel[:, 1], -rel[:, 0]])
    return sp.coo_matrix((sW, (iW, jW)), shape=(3 * nn, 6 * ngroups)).tocsr()


def dpcg(K, f, W, Minv, rtol=1e-8, maxIters=2000, shift=1e-10):
    """Deflated PCG of ``deflatedPCG_CPU`` (src/deflation.py:504-584).

    Dense symmetrised W^T K W + shift*I (:517-521), coarse start (:532-537),
    p0 = z - W mu (:542-549), stop on sqrt(r.z / r0.z0) <= rtol (:567).
    The coarse system is solved by a dense Cholesky factorisation.
    Returns (x, iterations).
    """
    WT = W.transpose().tocsr()
    KW = K @ W
    E = (WT @ KW).toarray()
    E = (E + E.T) / 2
    E += np.eye(E.shape[0]) * shift
    cf = sla.cho_factor(E, lower=True)

    def cs(v):
        return sla.cho_solve(cf, v)
    x = W @ cs(WT @ f)
    r = f - K @ x
    z = Minv * r
    p = z - W @ cs(WT @ (K @ z))
    rz = r.dot(z)
    rz0 = rz
    it = 0
    for it in range(maxIters):
        Kp = K @ p
        alpha = rz / p.dot(Kp)
        x += alpha * p
        r -= alpha * Kp
        z = Minv * r
        rz_new = r.dot(z)
        if np.sqrt(rz_new / rz0) <= rtol:
            break
        beta = rz_new / rz
        p = z + beta * p - W @ cs(WT @ (K @ z))
        rz = rz_new
    return x, it + 1


# --------------------------------------------------------------------------
# a8-a11: objectives and sensitivities (src/topopt_obj_cons_sensitivities.py)
# --------------------------------------------------------------------------
def compliance_and_gradient(u, x, edof, Ke, penal=3.0, emin=1e-8):
    """ce = u_e^T Ke u_e; C = sum s ce; dC = -ds ce
    (src/topopt_obj_cons_sensitivities.py:148-179)."""
    ue = u[edof]
    ce = (ue @ Ke * ue).sum(1)
    C = np.sum(simp_scaling(x, penal, emin) * ce)
    return C, -simp_sensitivity(x, penal, emin) * ce, ce


def _gradN(elem_size):
    g = (1 / 8) * np.array([[-1, 1, 1, -1, -1, 1, 1, -1],
                            [-1, -1, 1, 1, -1, -1, 1, 1],
                            [-1, -1, -1, -1, 1, 1, 1, 1]], dtype=float)
    for i in range(3):
        g[i, :] = 2 * g[i, :] / elem_size[i]
    return g


def postprocess(u, x, edof, E, nu, elem_size, q=0.5, P=6.0):
    """Centroid strain/stress, von Mises, p-norm, strain energy
    (src/hex_structural_fea.py:152-234).  Strain order xx,yy,zz,xy,xz,yz."""
    gN = _gradN(elem_size)
    uG = gN @ u[edof[:, 0::3]].T
    vG = gN @ u[edof[:, 1::3]].T
    wG = gN @ u[edof[:, 2::3]].T
    strain = np.stack([uG[0], vG[1], wG[2], uG[1] + vG[0], uG[2] + wG[0], vG[2] + wG[1]], axis=1)
    D = constitutive_matrix(E, nu)
    stress = np.einsum("ij,ej->ei", D, strain)
    stress *= (x ** q).reshape((-1, 1))
    s = stress
    vm = np.sqrt(0.5 * ((s[:, 0] - s[:, 1]) ** 2 + (s[:, 1] - s[:, 2]) ** 2 + (s[:, 2] - s[:, 0]) ** 2)
                 + 3 * (s[:, 3] ** 2 + s[:, 4] ** 2 + s[:, 5] ** 2))
    pnorm = (np.sum(vm ** P)) ** (1 / P)
    sed = 0.5 * np.sum(strain * stress, axis=1)
    return dict(strain=strain, stress=stress, vm=vm, pnorm=pnorm, sed=sed)


def _Bmat(elem_size):
    gN = _gradN(elem_size)
    Bi = np.zeros((6, 3, 8))
    Bi[0, 0, :] = gN[0]
    Bi[1, 1, :] = gN[1]
    Bi[2, 2, :] = gN[2]
    Bi[3, 0, :] = gN[1]
    Bi[3, 1, :] = gN[0]
    Bi[4, 0, :] = gN[2]
    Bi[4, 2, :] = gN[0]
    Bi[5, 1, :] = gN[2]
    Bi[5, 2, :] = gN[1]
    B = np.zeros((6, 24))
    idx = np.arange(8)
    B[:, (3 * idx)[:, None] + np.arange(3)] = Bi.transpose(0, 2, 1)
    return B


def pnorm_stress_and_sensitivity(u, x, edof, Ke, E, nu, elem_size, adjoint_solve,
                                 q=0.5, P=6.0, penal=3.0, emin=1e-8):
    """p-norm von Mises and its adjoint sensitivity
    (src/topopt_obj_cons_sensitivities.py:181-287), loops vectorised.

    ``adjoint_solve(g)`` must return K^-1 g with the same boundary conditions
    (the reference calls ``linear_solvers.solve`` at :269-274).
    """
    post = postprocess(u, x, edof, E, nu, elem_size, q, P)
    D = constitutive_matrix(E, nu)
    B = _Bmat(elem_size)
    vm = post["vm"]
    st = post["stress"]
    dpn = (np.sum(vm ** P)) ** (1 / P - 1)
    s11, s22, s33, s12, s13, s23 = (st[:, i] for i in range(6))
    DvmDs = np.stack([1 / (2 * vm) * (2 * s11 - s22 - s33), 1 / (2 * vm) * (2 * s22 - s11 - s33),
                      1 / (2 * vm) * (2 * s33 - s11 - s22), 3 / vm * s12, 3 / vm * s13, 3 / vm * s23], 1)
    xc = np.maximum(x, 1e-12)
    ue = u[edof]
    F = D @ B
    beta = (q * xc ** (q - 1)) * (vm ** (P - 1)) * np.einsum("ei,ij,ej->e", DvmDs, F, ue)
    T1 = dpn * beta
    ge = ((xc ** q) * dpn * (vm ** (P - 1)))[:, None] * (DvmDs @ F)  # (ne,24) = B^T D^T DvmDs
    g = np.zeros(u.shape[0])
    np.add.at(g, edof.ravel(), ge.ravel())
    lam = adjoint_solve(g)
    ce = (lam[edof] @ Ke * ue).sum(1)
    T2 = -simp_sensitivity(xc, penal, emin) * ce
    return post["pnorm"], T1 + T2, np.max(vm), dict(g=g, lam=lam, T1=T1, T2=T2)


def solution_dotproduct_and_gradient(u, x, edof, Ke, g, adjoint_solve, penal=3.0, emin=1e-8):
    """obj = u.g; lam = -K^-1 g; grad = ds * lam_e^T Ke u_e
    (src/topopt_obj_cons_sensitivities.py:289-319)."""
    obj = np.dot(u, g)
    lam = -adjoint_solve(g)
    ce = (lam[edof] @ Ke * u[edof]).sum(1)
    return obj, simp_sensitivity(x, penal, emin) * ce


# --------------------------------------------------------------------------
# a12/a14: smoothing filter (src/topopt_filters.py:8-38)
# --------------------------------------------------------------------------
def smoothing_filter(mesh: dict, rel_filter_radius: float = 1.5):
    """H_ij = (r - d_ij)/r for d_ij <= r, r = rel * elem_size[0]; Hs = row sums
    (src/topopt_filters.py:8-38).  Built from grid offsets instead of the
    reference's hash-grid loop; the element set and weights are the same."""
    nx, ny, nz = mesh["nelx"], mesh["nely"], mesh["nelz"]
    h = mesh["elem_size"]
    r = rel_filter_radius * h[0]
    R = [int(math.ceil(r / h[d])) + 1 for d in range(3)]
    ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    rows, cols, vals = [], [], []
    c = mesh["elem_centers"]
    for dz in range(-R[2], R[2] + 1):
        for dy in range(-R[1], R[1] + 1):
            for dx in range(-R[0], R[0] + 1):
                jx, jy, jz = ex + dx, ey + dy, ez + dz
                ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny) & (jz >= 0) & (jz < nz)
                i = np.where(ok)[0]
                j = jx[ok] + nx * (jy[ok] + ny * jz[ok])
                d = np.linalg.norm(c[i] - c[j], axis=1)
                keep = d <= r
                rows.append(i[keep])
                cols.append(j[keep])
                vals.append((r - d[keep]) / r)
    H = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(mesh["num_elems"],) * 2).tocsc()
    Hs = np.array(H.sum(1)).squeeze()
    return H, Hs


def mirror_filter(mesh: dict, axis: int) -> sp.csr_matrix:
    """Mirror-symmetry filter about the mid-plane normal to `axis` on a full box grid
    (createX/Y/ZSymmetryFilter, src/topopt_filters.py:292-393): row i holds 0.5 at i
    and 0.5 at its mirror element, or 1.0 at i when i is its own mirror."""
    n = (mesh["nelx"], mesh["nely"], mesh["nelz"])
    ne = mesh["num_elems"]
    e = np.arange(ne)
    ijk = [e % n[0], (e // n[0]) % n[1], e // (n[0] * n[1])]
    ijk[axis] = n[axis] - 1 - ijk[axis]
    m = ijk[0] + n[0] * (ijk[1] + n[1] * ijk[2])
    return (sp.coo_matrix((np.full(ne, 0.5), (e, e)), shape=(ne, ne))
            + sp.coo_matrix((np.full(ne, 0.5), (e, m)), shape=(ne, ne))).tocsr()


def extrude_filter(mesh: dict, axis: int) -> sp.csr_matrix:
    """Extrusion filter along `axis` on a full box grid (createX/Y/ZExtrudeFilter,
    src/topopt_filters.py:595-716): for each line of elements along axis, visited from
    its lowest element id, the matching elements are the whole line plus that first
    element once more, so with n elements per line and w = 1/(n+1) the summed COO
    entries are w between two other elements, 2w between the first and another, 4w
    on the first's diagonal."""
    n = (mesh["nelx"], mesh["nely"], mesh["nelz"])
    ne = mesh["num_elems"]
    stride = (1, n[0], n[0] * n[1])[axis]
    e = np.arange(ne)
    first = e[((e // stride) % n[axis]) == 0]
    rows, cols, vals = [], [], []
    w = 1.0 / (n[axis] + 1)
    for e0 in first:
        match = [e0 + t * stride for t in range(n[axis])] + [e0]
        for a in match:
            for b in match:
                rows.append(a)
                cols.append(b)
                vals.append(w)
    return sp.coo_matrix((vals, (rows, cols)), shape=(ne, ne)).tocsr()


# --------------------------------------------------------------------------
# a13: OC update and loop (src/topopt_ocm.py:107-345)
# --------------------------------------------------------------------------
def volume_constraint(x, volfrac):
    """(mean(x)/volfrac - 1, 1/volfrac/n) (src/topopt_obj_cons_sensitivities.py:100-116)."""
    return (np.mean(x) / volfrac) - 1.0, np.ones_like(x) / volfrac / x.size


def oc_update(x, grad, volfrac, move=0.2, xmin=0.001, xmax=1.0):
    """Bisection on the volume multiplier (src/topopt_ocm.py:251-269)."""
    _, dv = volume_constraint(x, volfrac)
    l1, l2 = 0.0, 1e12
    xnew = x
    while (l2 - l1) / ((l1 + l2) / 2 + 1e-10) > 1e-7:
        lmid = 0.5 * (l2 + l1)
        D = -grad / (dv * lmid)
        D = np.clip(D, 0.1, 10)
        xnew = np.maximum(xmin, np.maximum(x - move, np.minimum(xmax, np.minimum(x + move, x * np.sqrt(D)))))
        vc, _ = volume_constraint(xnew, volfrac)
        if vc > 0:
            l1 = lmid
        else:
            l2 = lmid
    return xnew


def elements_with_forces(mesh, force, ndof_per_node=3):
    """``find_elements_with_forces`` (src/topopt_common.py:79-100)."""
    forced_nodes = np.unique(np.where(force != 0)[0] // ndof_per_node)
    is_forced = np.isin(mesh["elemArray"], forced_nodes)
    return np.where(is_forced.any(axis=1))[0]


def topopt_oc(mesh, Ke, force, solve_fn, volfrac, n_iter, H, Hs, move=0.2, penal=3.0, emin=1e-8):
    """OC loop with sensitivity filter, normalised objective, loaded-element
    clamp (src/topopt_ocm.py:170-306).  ``solve_fn(x) -> u``.  Returns the
    objective history (un-normalised, :277) and the final x.  The
    binarisation / connected-component post-pass (:312-329) is not restated."""
    ne = mesh["num_elems"]
    x = volfrac * np.ones(ne)
    loaded = elements_with_forces(mesh, force)
    hist = []
    objScaling = None
    for _ in range(n_iter):
        u = solve_fn(x)
        obj, grad, _ = compliance_and_gradient(u, x, mesh["edof"], Ke, penal, emin)
        if objScaling is None:
            objScaling = abs(obj)
        obj = obj / objScaling
        grad = grad / objScaling
        grad = (H * (x * grad)) / Hs / x
        if loaded.size > 0:
            grad[loaded] = np.min(grad)
        x = oc_update(x, grad, volfrac, move)
        hist.append(obj * objScaling)
    return np.array(hist), x


def cantilever_bc(mesh: dict):
    """Config cantilever: all DOFs of ix=0 nodes fixed; unit total -z load split
    over the ix=nelx, iz=0 edge nodes (pattern of src/hex_structural_examples.py:665-669)."""
    ni = mesh["node_indices"]
    fixed_nodes = np.where(ni[:, 0] == 0)[0]
    fixed = np.sort(np.concatenate([3 * fixed_nodes + c for c in range(3)]))
    load_nodes = np.where((ni[:, 0] == mesh["nelx"]) & (ni[:, 2] == 0))[0]
    f = np.zeros(3 * mesh["num_nodes"])
    f[3 * load_nodes + 2] = -1.0 / len(load_nodes)
    return f, fixed.astype(np.int64)
