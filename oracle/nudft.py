"""FP64 direct non-uniform DFT -- the definition the reference's NUFFT calls compute.

Conventions of cpp/corelib/lib/fft/nufft.cppm: coords[i] pairs with image dimension i (the
reference reverses them for cufinufft's fastest-first order, :191-199), centred mode order
(mode index i <-> k = i - floor(N/2)), type-1 sign +1, type-2 sign -1 (:50-55):

    type 1:  f[k] = sum_j c_j exp(+i s k.x_j)       (c: [T, M] -> f: [T, N0, ..])
    type 2:  c_j  = sum_k f[k] exp(+i s k.x_j)      (f: [T, N0, ..] -> c: [T, M])
"""
from __future__ import annotations

import numpy as np


def modes(N: int) -> np.ndarray:
    return np.arange(N, dtype=np.float64) - (N // 2)


def _phase(N: int, x: np.ndarray, sign: int) -> np.ndarray:
    # [N, M]
    return np.exp(1j * sign * np.outer(modes(N), x.astype(np.float64)))


def type1(coords, c, nmodes, sign: int = 1, chunk: int = 4096) -> np.ndarray:
    c = np.asarray(c, dtype=np.complex128)
    T, M = c.shape
    dim = len(nmodes)
    out = np.zeros((T, *nmodes), dtype=np.complex128)
    for j0 in range(0, M, chunk):
        sl = slice(j0, min(M, j0 + chunk))
        E = [_phase(nmodes[i], np.asarray(coords[i])[sl], sign) for i in range(dim)]
        cc = c[:, sl]
        if dim == 1:
            out += cc @ E[0].T
        elif dim == 2:
            # f[t, a, b] = sum_j c[t,j] E0[a,j] E1[b,j]
            out += np.einsum("tj,aj,bj->tab", cc, E[0], E[1], optimize=True)
        else:
            for a in range(nmodes[0]):
                w = cc * E[0][a][None, :]                      # [T, m]
                # [T, N1, N2] = sum_j w[t,j] E1[b,j] E2[c,j]
                out[:, a] += np.einsum("tj,bj,cj->tbc", w, E[1], E[2], optimize=True)
    return out


def type2(coords, f, sign: int = -1, chunk: int = 2048) -> np.ndarray:
    f = np.asarray(f, dtype=np.complex128)
    T = f.shape[0]
    nmodes = f.shape[1:]
    dim = len(nmodes)
    M = np.asarray(coords[0]).shape[0]
    out = np.zeros((T, M), dtype=np.complex128)
    for j0 in range(0, M, chunk):
        sl = slice(j0, min(M, j0 + chunk))
        E = [_phase(nmodes[i], np.asarray(coords[i])[sl], sign) for i in range(dim)]
        if dim == 1:
            out[:, sl] = f @ E[0]
        elif dim == 2:
            t = np.einsum("tab,bj->taj", f, E[1], optimize=True)
            out[:, sl] = np.einsum("taj,aj->tj", t, E[0], optimize=True)
        else:
            t = np.einsum("tabc,cj->tabj", f, E[2], optimize=True)
            t = np.einsum("tabj,bj->taj", t, E[1], optimize=True)
            out[:, sl] = np.einsum("taj,aj->tj", t, E[0], optimize=True)
    return out


def type1_at(coords, c, nmodes, idx, sign: int = 1) -> np.ndarray:
    """Type-1 at selected mode indices idx ([K, dim] ints) only: spot checks at full size."""
    c = np.asarray(c, dtype=np.complex128)
    idx = np.asarray(idx)
    ph = np.zeros((idx.shape[0], np.asarray(coords[0]).shape[0]))
    for i in range(len(nmodes)):
        k = idx[:, i].astype(np.float64) - nmodes[i] // 2
        ph += np.outer(k, np.asarray(coords[i], dtype=np.float64))
    return c @ np.exp(1j * sign * ph).T  # [T, K]


def type2_at(coords, f, pts, sign: int = -1) -> np.ndarray:
    """Type-2 at selected points only (pts: indices into the coordinate arrays)."""
    f = np.asarray(f, dtype=np.complex128)
    nmodes = f.shape[1:]
    sub = [np.asarray(c, dtype=np.float64)[pts] for c in coords]
    return type2(sub, f, sign=sign)
