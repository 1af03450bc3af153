"""Generates the committed golden fixtures of tests/golden/ (run from the repository root:
``python tests/golden/make_golden.py``). Needs oracle/_ref/libref_toeplitz_load.so, i.e. the
reference's own Toeplitz load/store kernels built by oracle/ref_load/Makefile.

Fixtures
--------
nudft_{1d,2d,3d}.npz   FP64 direct NUDFT type 1 / type 2 (the definition the reference's
                       cufinufft calls compute: nufft.cppm:50-55, 191-199, centred modes).
ref_toeplitz_{2d,3d}.npz  inputs and outputs of the reference's toeplitz_load_2D/3D kernels
                       (cpp/corelib/lib/fft/kernels/) driven through the reference's
                       multiplication sequence (fft/toeplitz.cppm:232-501) with the straight
                       convolution between launches, for several multiply-flag sets.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import nudft, refload  # noqa: E402

OUT = Path(__file__).resolve().parent
FLAGS = np.array([(0, 1, 2, 1, 2, 0), (2, 1, 0, 0, 0, 0), (0, 1, 2, 0, 0, 0), (1, 2, 1, 2, 1, 1), (0, 0, 0, 0, 0, 1)],
                 dtype=np.int32)


def crand(rng, *shape):
    return ((rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)).astype(np.complex64)


def make_nudft(dim, nmodes, M, T, seed):
    rng = np.random.default_rng(seed)
    coords = np.stack([rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]).astype(np.float32)
    c = crand(rng, T, M)
    f = crand(rng, T, *nmodes)
    t1 = nudft.type1(list(coords), c, nmodes, sign=1)
    t2 = nudft.type2(list(coords), f, sign=-1)
    np.savez_compressed(OUT / f"nudft_{dim}d.npz", coords=coords, c=c, f=f, type1=t1.astype(np.complex128),
                        type2=t2.astype(np.complex128), nmodes=np.array(nmodes))


def make_ref(dim, shape, B, seed):
    if not refload.available():
        raise SystemExit("oracle/_ref/libref_toeplitz_load.so missing: run make -C oracle/ref_load")
    rng = np.random.default_rng(seed)
    inp = crand(rng, B, *shape)
    out0 = crand(rng, B, *shape)
    m1 = crand(rng, *shape)
    m2 = crand(rng, *shape)
    K = crand(rng, *[2 * s for s in shape])
    outs = []
    for fl in FLAGS:
        io, i1, o1, i2, o2, acc = (int(v) for v in fl)
        outs.append(refload.multiplication(inp, out0, K.astype(np.complex128), m1, m2, io, i1, o1, i2, o2, acc))
    np.savez_compressed(OUT / f"ref_toeplitz_{dim}d.npz", input=inp, out0=out0, mult1=m1, mult2=m2, kernel=K,
                        flags=FLAGS, outputs=np.stack(outs))


if __name__ == "__main__":
    make_nudft(1, (24,), 300, 2, 1)
    make_nudft(2, (12, 10), 600, 2, 2)
    make_nudft(3, (8, 10, 6), 800, 2, 3)
    make_ref(3, (6, 8, 10), 2, 4)
    make_ref(2, (10, 12), 3, 5)
    for p in sorted(OUT.glob("*.npz")):
        print(p.name, p.stat().st_size)
