"""Synthetic HCurl (lowest-order Nedelec) systems on a Kuhn tetrahedral mesh.

Stands in for the NGSolve assembly behind the reference's AMS benchmarks
(examples/hiruma/*.py use meshes that are not available): the unit cube cut
into nc^3 cubes, each split into 6 tetrahedra around its main diagonal (Kuhn
subdivision); Whitney edge elements w_ab = l_a grad l_b - l_b grad l_a with
edges oriented from the lower to the higher vertex number; the discrete
gradient G (+1 at the higher vertex, -1 at the lower one); vertex
coordinates; element-wise material coefficients; Dirichlet on every edge of
the boundary surface; and a source made of closed edge loops, so that
G^T f = 0 exactly (a discretely divergence-free current).

Sizes: nc = 40 gives 68,921 vertices and 462,520 edges; nc = 64 gives
274,625 vertices and 1,872,064 edges.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

NU0 = 1.0 / (4e-7 * np.pi)  # reluctivity of vacuum (SI)

# local edges of a tetrahedron (vertex pairs)
_LE = np.array([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)])


@dataclass
class KuhnMesh:
    nc: int
    coords: np.ndarray      # (nv, 3)
    tets: np.ndarray        # (nt, 4) vertex ids
    edges: np.ndarray       # (ne, 2) vertex ids, low -> high
    tet_edges: np.ndarray   # (nt, 6) edge ids of the local edges _LE
    tet_signs: np.ndarray   # (nt, 6) +1 if the local edge runs low -> high
    centroids: np.ndarray   # (nt, 3)
    grads: np.ndarray       # (nt, 4, 3) barycentric gradients
    vol: np.ndarray         # (nt,)

    @property
    def nv(self):
        return self.coords.shape[0]

    @property
    def ne(self):
        return self.edges.shape[0]


def kuhn_mesh(nc: int) -> KuhnMesh:
    n1 = nc + 1
    g = np.arange(n1, dtype=np.float64) / nc
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    coords = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)

    def vid(i, j, k):
        return i + n1 * (j + n1 * k)

    ii, jj, kk = np.meshgrid(np.arange(nc), np.arange(nc), np.arange(nc), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    tets = []
    unit = np.eye(3, dtype=np.int64)
    for perm in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
        off = np.zeros(3, dtype=np.int64)
        vs = [vid(ii, jj, kk)]
        for ax in perm:
            off = off + unit[ax]
            vs.append(vid(ii + off[0], jj + off[1], kk + off[2]))
        tets.append(np.stack(vs, axis=1))
    tets = np.concatenate(tets, axis=0).astype(np.int64)
    nt = tets.shape[0]
    a = tets[:, _LE[:, 0]]
    b = tets[:, _LE[:, 1]]
    lo = np.minimum(a, b)
    hi = np.maximum(a, b)
    key = lo * n1 ** 3 + hi
    ukey, inv = np.unique(key.ravel(), return_inverse=True)
    edges = np.stack([ukey // n1 ** 3, ukey % n1 ** 3], axis=1)
    tet_edges = inv.reshape(nt, 6)
    tet_signs = np.where(a < b, 1.0, -1.0)
    P = coords[tets]  # (nt, 4, 3)
    J = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2)  # columns
    det = np.linalg.det(J)
    Jinv = np.linalg.inv(J)  # rows = grad l1..l3
    grads = np.zeros((nt, 4, 3))
    grads[:, 1:, :] = Jinv
    grads[:, 0, :] = -Jinv.sum(axis=1)
    return KuhnMesh(nc, coords, tets, edges, tet_edges, tet_signs, P.mean(axis=1), grads, np.abs(det) / 6.0)


def element_matrices(m: KuhnMesh):
    """Whitney curl-curl (per unit nu) and mass element matrices, (nt,6,6)."""
    ga = m.grads[:, _LE[:, 0], :]  # (nt,6,3)
    gb = m.grads[:, _LE[:, 1], :]
    s = m.tet_signs[:, :, None]
    curl = 2.0 * np.cross(ga, gb) * s  # (nt,6,3)
    Ke = np.einsum("tie,tje->tij", curl, curl) * m.vol[:, None, None]
    # int l_a l_b = vol (1 + delta_ab) / 20
    G = np.einsum("tae,tbe->tab", m.grads, m.grads)  # grad l_a . grad l_b (nt,4,4)
    I = (np.ones((4, 4)) + np.eye(4)) / 20.0
    i, j = _LE[:, 0], _LE[:, 1]
    Me = (I[np.ix_(i, i)][None] * G[:, j][:, :, j]
          - I[np.ix_(i, j)][None] * G[:, j][:, :, i]
          - I[np.ix_(j, i)][None] * G[:, i][:, :, j]
          + I[np.ix_(j, j)][None] * G[:, i][:, :, i])
    Me = Me * m.vol[:, None, None] * (s * np.swapaxes(s, 1, 2))
    return Ke, Me


def assemble(m: KuhnMesh, coef_e: np.ndarray, Ee: np.ndarray, dtype=np.float64):
    """sum_t coef_t * E_t scattered to edges; CSR, sorted, duplicates summed."""
    rows = np.repeat(m.tet_edges, 6, axis=1).ravel()
    cols = np.tile(m.tet_edges, (1, 6)).ravel()
    vals = (Ee * coef_e[:, None, None]).reshape(-1).astype(dtype)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(m.ne, m.ne)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    A.indptr = A.indptr.astype(np.int32)
    A.indices = A.indices.astype(np.int32)
    return A


def gradient_matrix(m: KuhnMesh):
    """Discrete gradient G (ne x nv): +1 at the higher vertex, -1 at the lower."""
    ne = m.ne
    rows = np.repeat(np.arange(ne), 2)
    cols = m.edges.ravel()
    vals = np.tile([-1.0, 1.0], ne)
    G = sp.csr_matrix((vals, (rows, cols)), shape=(ne, m.nv))
    G.sort_indices()
    G.indptr = G.indptr.astype(np.int32)
    G.indices = G.indices.astype(np.int32)
    return G


def assemble_on_device(m: KuhnMesh, nu_e=None, kappa_e=None):
    """K = sum_t nu_t Ke_t, M = sum_t kappa_t Me_t and G assembled on the GPU
    (ssv_hcurl_assemble; nu_e / kappa_e None = 1), returned as scipy CSR
    matrices with the same patterns as assemble() and gradient_matrix()."""
    import ctypes

    from . import _capi
    lib = _capi.load()
    xyz = np.ascontiguousarray(m.coords, dtype=np.float64)
    tets = np.ascontiguousarray(m.tets, dtype=np.int32)
    te = np.ascontiguousarray(m.tet_edges, dtype=np.int32)
    sg = np.ascontiguousarray(m.tet_signs, dtype=np.int8)
    ev = np.ascontiguousarray(m.edges, dtype=np.int32)
    nu = None if nu_e is None else np.ascontiguousarray(nu_e, dtype=np.float64)
    ka = None if kappa_e is None else np.ascontiguousarray(kappa_e, dtype=np.float64)
    hs = [ctypes.c_void_p() for _ in range(3)]
    _capi.check(lib.ssv_hcurl_assemble(m.nv, _capi.vptr(xyz), tets.shape[0], _capi.vptr(tets), _capi.vptr(te),
                                       _capi.vptr(sg), m.ne, _capi.vptr(ev),
                                       None if nu is None else _capi.vptr(nu), None if ka is None else _capi.vptr(ka),
                                       ctypes.byref(hs[0]), ctypes.byref(hs[1]), ctypes.byref(hs[2])))
    out = []
    try:
        for h, ncols in zip(hs, (m.ne, m.ne, m.nv)):
            rows, cols, nnz, dt = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int32()
            _capi.check(lib.ssv_matrix_info(h, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(nnz),
                                            ctypes.byref(dt)))
            ip = np.empty(rows.value + 1, dtype=np.int32)
            ix = np.empty(nnz.value, dtype=np.int32)
            v = np.empty(nnz.value, dtype=np.float64)
            _capi.check(lib.ssv_matrix_export(h, _capi.vptr(ip), _capi.vptr(ix), _capi.vptr(v)))
            out.append(sp.csr_matrix((v, ix, ip), shape=(rows.value, ncols)))
    finally:
        for h in hs:
            if h.value:
                lib.ssv_matrix_destroy(h)
    return tuple(out)


def boundary_freedofs(m: KuhnMesh):
    """1 for free edges, 0 for edges lying in the boundary surface."""
    c = m.coords
    on = [(np.isclose(c[:, d], 0.0), np.isclose(c[:, d], 1.0)) for d in range(3)]
    a, b = m.edges[:, 0], m.edges[:, 1]
    bnd = np.zeros(m.ne, dtype=bool)
    for lo, hi in on:
        bnd |= (lo[a] & lo[b]) | (hi[a] & hi[b])
    return (~bnd).astype(np.uint8)


def loop_source(m: KuhnMesh, z_levels=(0.5,), squares=((0.15, 0.85),), scale=1.0):
    """Unit currents around closed squares of grid edges in z planes."""
    nc = m.nc
    n1 = nc + 1
    f = np.zeros(m.ne)
    key = m.edges[:, 0] * n1 ** 3 + m.edges[:, 1]
    order = np.argsort(key)
    ks = key[order]

    def edge(v0, v1):
        lo, hi = min(v0, v1), max(v0, v1)
        p = np.searchsorted(ks, lo * n1 ** 3 + hi)
        return order[p], (1.0 if v1 > v0 else -1.0)

    def vid(i, j, k):
        return i + n1 * (j + n1 * k)

    for z in z_levels:
        k = int(round(z * nc))
        for a0, b0 in squares:
            i0, i1 = int(round(a0 * nc)), int(round(b0 * nc))
            path = ([(i, i0) for i in range(i0, i1)] + [(i1, j) for j in range(i0, i1)] +
                    [(i, i1) for i in range(i1, i0, -1)] + [(i0, j) for j in range(i1, i0, -1)])
            pts = path + [path[0]]
            for (x0, y0), (x1, y1) in zip(pts[:-1], pts[1:]):
                e, sg = edge(vid(x0, y0, k), vid(x1, y1, k))
                f[e] += scale * sg
    return f


def _inside(c, lo, hi):
    return np.all((c >= lo) & (c <= hi), axis=1)


def magnetostatic(nc: int, nu_iron: float = 1e-3, mass_eps: float = 1e-6):
    """Configuration of the real AMS benchmark: nu = 1 in air, nu_iron in the
    centred 0.4^3 block [0.3, 0.7]^3, K + mass_eps * nu * M, loop source at
    mid-height around the block. Returns a dict of the system pieces."""
    m = kuhn_mesh(nc)
    Ke, Me = element_matrices(m)
    nu = np.where(_inside(m.centroids, 0.3, 0.7), nu_iron, 1.0)
    A = assemble(m, nu, Ke + mass_eps * Me)
    G = gradient_matrix(m)
    fd = boundary_freedofs(m)
    f = loop_source(m, z_levels=(0.5,), squares=((0.15, 0.85), (0.2, 0.8)))
    f = f * fd
    return dict(mesh=m, A=A, G=G, freedofs=fd, f=f, nu=nu, Ke=Ke, Me=Me,
                coords=(m.coords[:, 0].copy(), m.coords[:, 1].copy(), m.coords[:, 2].copy()))


def eddy_current(nc: int, freq: float = 3e4, sigma: float = 5.8e7, nu_r_core: float = 1e-3,
                 mass_eps: float = 1e-6):
    """Complex eddy-current configuration: A = K(nu) + j omega sigma M_cond,
    nu = nu0 * nu_r (nu_r = 1e-3 in the centred core [0.35,0.65]^3), sigma in a
    copper square annulus ([0.2,0.8]^2 minus [0.3,0.7]^2, z in [0.4,0.6]);
    auxiliary real SPD matrix a_real = K + |omega| sigma M_cond + mass_eps nu M.
    Loop source in air at mid-height outside the annulus."""
    m = kuhn_mesh(nc)
    Ke, Me = element_matrices(m)
    c = m.centroids
    core = _inside(c, 0.35, 0.65)
    ring = (_inside(c, np.array([0.2, 0.2, 0.4]), np.array([0.8, 0.8, 0.6]))
            & ~_inside(c, np.array([0.3, 0.3, 0.4]), np.array([0.7, 0.7, 0.6])))
    nu = NU0 * np.where(core, nu_r_core, 1.0)
    sig = np.where(ring, sigma, 0.0)
    omega = 2.0 * np.pi * freq
    K = assemble(m, nu, Ke)
    Mc = assemble(m, sig, Me)
    Mn = assemble(m, nu, Me)
    A = (K.astype(np.complex128) + 1j * omega * Mc.astype(np.complex128) + mass_eps * Mn).tocsr()
    a_real = (K + abs(omega) * Mc + mass_eps * Mn).tocsr()
    for X in (A, a_real):
        X.sort_indices()
        X.indptr = X.indptr.astype(np.int32)
        X.indices = X.indices.astype(np.int32)
    G = gradient_matrix(m)
    fd = boundary_freedofs(m)
    f = loop_source(m, z_levels=(0.5,), squares=((0.1, 0.9), (0.15, 0.85))) * fd
    return dict(mesh=m, A=A, a_real=a_real, G=G, freedofs=fd, f=f.astype(np.complex128), omega=omega,
                coords=(m.coords[:, 0].copy(), m.coords[:, 1].copy(), m.coords[:, 2].copy()))


def _eddy_fields(m: KuhnMesh, sigma: float, nu_r_core: float):
    c = m.centroids
    core = _inside(c, 0.35, 0.65)
    ring = (_inside(c, np.array([0.2, 0.2, 0.4]), np.array([0.8, 0.8, 0.6]))
            & ~_inside(c, np.array([0.3, 0.3, 0.4]), np.array([0.7, 0.7, 0.6])))
    return NU0 * np.where(core, nu_r_core, 1.0), np.where(ring, sigma, 0.0)


def _csr32(X):
    X = X.tocsr()
    X.sort_indices()
    X.indptr = X.indptr.astype(np.int32)
    X.indices = X.indices.astype(np.int32)
    return X


def eddy_family(nc: int, freqs=None, nrhs: int = 4, seed: int = 1, sigma: float = 5.8e7,
                nu_r_core: float = 1e-3, mass_eps: float = 1e-6):
    """Frequency family of the eddy-current configuration for batched solves:
    A_f = K + mass_eps nu M + j omega_f sigma M_cond = Kr + j omega_f Mc for
    freqs (default 8 log-spaced from 1 kHz to 100 kHz), a_real_f = K +
    |omega_f| sigma M_cond + mass_eps nu M per frequency, and nrhs source
    patterns (random square current loops in air: height, extent and amplitude
    drawn from numpy.random.default_rng(seed), snapped to interior grid lines)
    shared by every frequency.
    Returns Kr, Mc (real CSR), omegas, the per-frequency A and a_real, G,
    freedofs, coordinates and B of shape (F, nrhs, ne) complex."""
    freqs = np.logspace(3, 5, 8) if freqs is None else np.asarray(freqs, dtype=np.float64)
    m = kuhn_mesh(nc)
    Ke, Me = element_matrices(m)
    nu, sig = _eddy_fields(m, sigma, nu_r_core)
    K = assemble(m, nu, Ke)
    Mc = assemble(m, sig, Me)
    Mn = assemble(m, nu, Me)
    Kr = _csr32(K + mass_eps * Mn)
    omegas = 2.0 * np.pi * freqs
    A = [_csr32(K.astype(np.complex128) + 1j * w * Mc.astype(np.complex128) + mass_eps * Mn) for w in omegas]
    a_real = [_csr32(K + abs(w) * Mc + mass_eps * Mn) for w in omegas]
    fd = boundary_freedofs(m)
    rng = np.random.default_rng(seed)
    src = []
    for _ in range(nrhs):
        z = rng.uniform(0.25, 0.75)
        a0, b0 = rng.uniform(0.05, 0.15), rng.uniform(0.85, 0.95)
        amp = rng.uniform(0.5, 2.0)
        # snap to interior grid lines: a loop touching the boundary would be cut by the
        # Dirichlet mask and lose its zero divergence
        z = min(max(round(z * nc), 1), nc - 1) / nc
        a0 = max(round(a0 * nc), 1) / nc
        b0 = min(round(b0 * nc), nc - 1) / nc
        src.append(loop_source(m, z_levels=(z,), squares=((a0, b0),), scale=amp) * fd)
    B = np.broadcast_to(np.asarray(src, dtype=np.complex128), (len(omegas), nrhs, m.ne)).copy()
    return dict(mesh=m, K=Kr, M=_csr32(Mc), omegas=omegas, freqs=freqs, A=A, a_real=a_real,
                G=gradient_matrix(m), freedofs=fd, B=B,
                coords=(m.coords[:, 0].copy(), m.coords[:, 1].copy(), m.coords[:, 2].copy()))
