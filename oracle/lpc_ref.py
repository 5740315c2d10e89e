"""CPU reference of the learned preconditioner's data path (test
infrastructure only: it checks the library's device kernels in csrc/lpc.cu).

Per element i: its 16 nearest elements by centroid distance (itself first;
scipy's k-d tree), then per neighbour j the centroid offset and normal in i's
(normal, strike, dip) frame -- the offset divided by h_i = sqrt(2 area_i) --
and the area ratio area_j / area_i (112 inputs); the training targets are the
3 x 3 blocks (A^-1)[i, j] (rows i, N + i, 2N + i; columns j, N + j, 2N + j)
divided by h_i / G.  Frames as the reference's CalculateSSandDSDirs
(src/CalculateSSandDSDirs.jl:42-98) and triangle normals as
CreateFaceNormalAndMidPoint (src/CreateFaceNormalAndMidPoint.jl:66-115).
"""
import numpy as np

K = 16
N_IN = 7 * K
N_OUT = 9 * K


def _ss_ds(cx, cy, cz):
    with np.errstate(invalid="ignore", divide="ignore"):
        nrm = np.sqrt(cx * cx + cy * cy)
        r1, r2 = cx / nrm, cy / nrm
    ss = np.stack([-r2, r1, np.zeros_like(cx)], axis=1)
    dsz = np.cos(np.arccos(cz) - np.pi / 2)
    L = np.sin(np.arccos(dsz))
    L = np.where(cz < 0, -L, L)
    a = np.arctan2(cy, cx)
    ds = np.stack([-np.cos(a) * L, -np.sin(a) * L, dsz], axis=1)
    vert = (cx == 0) & (cy == 0)
    ds[vert] = [-1.0, 0.0, 0.0]
    ss[vert & (cz < 1.0)] = [0.0, -1.0, 0.0]
    ss[vert & ~(cz < 1.0)] = [0.0, 1.0, 0.0]
    return ss, ds


def element_frames(P1, P2, P3):
    """Centroids, unit normals, strike and dip directions, areas."""
    P1, P2, P3 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (P1, P2, P3))
    w = np.cross(P2 - P1, P3 - P1)
    ln = np.sqrt((w * w).sum(1))
    nrm = w / ln[:, None]
    ss, ds = _ss_ds(nrm[:, 0], nrm[:, 1], nrm[:, 2])
    return (P1 + P2 + P3) / 3.0, nrm, ss, ds, 0.5 * ln


def features(P1, P2, P3):
    """(X, nbr, h): inputs (N x 112, float32), neighbours (N x 16, int32,
    itself first; meshes of fewer than 16 elements repeat the farthest) and
    h = sqrt(2 area)."""
    from scipy.spatial import cKDTree
    cen, nrm, ss, ds, area = element_frames(P1, P2, P3)
    n = len(cen)
    k = min(K, n)
    nbr = cKDTree(cen).query(cen, k=k)[1].reshape(n, k)
    if k < K:
        nbr = np.concatenate([nbr, np.repeat(nbr[:, -1:], K - k, axis=1)], axis=1)
    h = np.sqrt(2.0 * area)
    R = np.stack([nrm, ss, ds], axis=1)
    off = np.einsum("iab,ikb->ika", R, cen[nbr] - cen[:, None, :]) / h[:, None, None]
    nloc = np.einsum("iab,ikb->ika", R, nrm[nbr])
    arat = (area[nbr] / area[:, None])[..., None]
    X = np.concatenate([off, nloc, arat], axis=2).reshape(n, N_IN)
    return X.astype(np.float32), nbr.astype(np.int32), h


def inverse_blocks(Ainv, nbr, h, G):
    """Targets (N x 144): (A^-1)[i, nbr[i, q]] blocks divided by h_i / G."""
    n = nbr.shape[0]
    rows = np.stack([np.arange(n), n + np.arange(n), 2 * n + np.arange(n)], axis=1)
    cols = np.stack([nbr, n + nbr, 2 * n + nbr], axis=2)
    T = Ainv[rows[:, None, :, None], cols[:, :, None, :]]
    return (T / (h / G)[:, None, None, None]).reshape(n, N_OUT).astype(np.float32)
