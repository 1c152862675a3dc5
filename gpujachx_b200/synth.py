"""Seeded synthetic inputs of the benchmark configurations (no dataset exists).

Every generator returns a Fortran-ordered float64 (m, n) array; the same seed
gives the same bits on any host with this numpy (BLAS calls are pinned to one
thread while generating so that the QR factors are reproducible).

* :func:`gaussian`  -- i.i.d. N(0,1) entries (config 2: 4096 x 2048)
* :func:`svd_synth` -- Q1 diag(s) Q2^T, Haar Q1/Q2, s geometric from 1 to smin
                       (configs 1 and 4, the batch of config 5)
* :func:`graded`    -- B diag(d), B i.i.d. N(0,1), d_j = 10^U(lo, 0) (config 3)
* :func:`haar_gpu`  -- Q1 diag(s) Q2^T formed on the GPU (torch CUDA generator):
                       the 8192 x 8192 configuration is too large for a host QR
                       at start-up; the same seed gives the same bits with the
                       same torch / CUDA build on a B200
"""

from __future__ import annotations

import hashlib

import numpy as np

try:
    from threadpoolctl import threadpool_limits
except ImportError:  # pragma: no cover
    threadpool_limits = None


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def gaussian(m: int, n: int, seed: int) -> np.ndarray:
    return np.asfortranarray(_rng(seed).standard_normal((n, m)).T)


def _haar(rng: np.random.Generator, n: int) -> np.ndarray:
    Z = rng.standard_normal((n, n))
    Q, R = np.linalg.qr(Z)
    return Q * np.sign(np.diag(R))


def svd_synth(m: int, n: int, seed: int, smin: float = 1e-8) -> np.ndarray:
    rng = _rng(seed)
    s = np.geomspace(1.0, smin, n) if n > 1 else np.ones(1)

    def go():
        Q1 = _haar(rng, m)[:, :n]
        Q2 = _haar(rng, n)
        return np.asfortranarray((Q1 * s) @ Q2.T)

    if threadpool_limits is not None:
        with threadpool_limits(limits=1):
            return go()
    return go()


def graded(m: int, n: int, seed: int, lo: float = -6.0) -> np.ndarray:
    rng = _rng(seed)
    B = rng.standard_normal((n, m)).T
    d = 10.0 ** rng.uniform(lo, 0.0, n)
    return np.asfortranarray(B * d)


def haar_gpu(m: int, n: int, seed: int, smin: float = 1e-12) -> np.ndarray:
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    def haar(k):
        q, r = torch.linalg.qr(torch.randn((k, k), dtype=torch.float64, device=dev, generator=gen))
        return q * torch.sign(torch.diagonal(r)).unsqueeze(0)

    sv = torch.logspace(0.0, float(np.log10(smin)), n, dtype=torch.float64, device=dev)
    G = (haar(m)[:, :n] * sv) @ haar(n).T
    return np.asfortranarray(G.cpu().numpy())


def digest(a) -> str:
    """sha256 of the bytes of a float64 array in Fortran order."""
    return hashlib.sha256(np.asfortranarray(a, dtype=np.float64).tobytes(order="F")).hexdigest()


GENERATORS = {"gaussian": gaussian, "svd_synth": svd_synth, "graded": graded, "haar_gpu": haar_gpu}


def make(gen: str, m: int, n: int, seed: int, **kw) -> np.ndarray:
    return GENERATORS[gen](m, n, seed, **kw)
