"""Host restatement of the STOMP noise and metric operators, the checker of
the device loop (tests only).

* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
  easy as 1, 2, 3", SC 2011), pinned by the known-answer vectors of the
  paper's reference implementation (tests/test_stomp_host.py).
* Box-Muller on the top 24 bits of each word, FP64.
* R (chomp_precompute.cpp:20-37 / stomp_precompute.cpp:24-42), the dense
  Cholesky factor L of the rescaled inverse (stomp_precompute.cpp:46-68) and
  the column-scaled projection M (stomp_precompute.cpp:70-94), FP64.
"""
import numpy as np

from prismplan_b200 import workloads


def philox4x32_10(c, k0, k1):
    """Philox4x32-10 (Salmon et al., SC 2011) on uint32 counters c[4]."""
    m = np.uint64(0xFFFFFFFF)
    c = [np.asarray(x, np.uint64) & m for x in c]
    k0, k1 = np.uint64(k0), np.uint64(k1)
    for _ in range(10):
        p0 = np.uint64(0xD2511F53) * c[0]
        p1 = np.uint64(0xCD9E8D57) * c[2]
        c = [((p1 >> np.uint64(32)) ^ c[1] ^ k0) & m, p1 & m, ((p0 >> np.uint64(32)) ^ c[3] ^ k1) & m, p0 & m]
        k0 = (k0 + np.uint64(0x9E3779B9)) & m
        k1 = (k1 + np.uint64(0xBB67AE85)) & m
    return c


def normals(rows, D, T, step, seed):
    """z [len(rows), D, T] of the device stream: counter (t // 4, r * D + d,
    step, 0), Box-Muller on the top 24 bits of each word, FP64."""
    rows = np.asarray(rows)
    nk = (T + 3) // 4
    r, d, k = np.meshgrid(rows, np.arange(D), np.arange(nk), indexing="ij")
    o = philox4x32_10([k, r * D + d, np.full_like(k, step), np.zeros_like(k)], seed & 0xFFFFFFFF, seed >> 32)
    u = [((x >> np.uint64(8)).astype(np.float64) + 0.5) * 2.0 ** -24 for x in o]
    z = np.empty(r.shape + (4,))
    for a, bb, j in ((u[0], u[1], 0), (u[2], u[3], 2)):
        rad = np.sqrt(-2.0 * np.log(a))
        z[..., j] = rad * np.cos(2 * np.pi * bb)
        z[..., j + 1] = rad * np.sin(2 * np.pi * bb)
    return z.reshape(len(rows), D, nk * 4)[:, :, :T]


def stomp_matrices(T, dt, noise_scale):
    """R, L (stomp_precompute.cpp:46-68) and M (:70-94), FP64."""
    R = workloads.control_cost_R(T, dt)
    Rinv = np.linalg.inv(R + 1e-8 * np.eye(T))
    S = Rinv * ((1.0 / T) / max(Rinv.max(), 1e-12))
    S = 0.5 * (S + S.T)
    L = np.linalg.cholesky(S) * noise_scale
    M = Rinv * ((1.0 / T) / np.maximum(Rinv.max(0), 1e-12))[None, :]
    return R, L, M
