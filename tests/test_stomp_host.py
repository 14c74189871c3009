"""The host restatement used to check the device STOMP loop, pinned on the
CPU: Philox4x32-10 against the published known-answer vectors, the normal
variates' moments, and the banded form of the noise factor and projection
that the device applies (L = sqrt(c) J Lb^-T J, M x = (R + 1e-8 I)^-1 (s .* x))
against the dense matrices of stomp_precompute.cpp:46-94."""
import numpy as np

from prismplan_b200 import workloads
from stomp_host import normals, philox4x32_10, stomp_matrices

# (counter, key) -> output, Philox4x32-10 known-answer vectors of the
# reference implementation accompanying Salmon et al. (SC 2011)
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def test_philox_known_answers():
    for ctr, key, want in KAT:
        got = philox4x32_10([np.array([c]) for c in ctr], *key)
        assert tuple(int(x[0]) for x in got) == want


def test_normals_moments():
    z = normals(np.arange(64), 7, 100, 3, 0x5BE5)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
    assert abs(np.corrcoef(z[:, :, :-1].ravel(), z[:, :, 1:].ravel())[0, 1]) < 0.01


def test_banded_forms_equal_dense_matrices():
    for T in (2, 7, 51, 100):
        R, L, M = stomp_matrices(T, 0.1, 1.0)
        A = R + 1e-8 * np.eye(T)
        Lb = np.linalg.cholesky(A)
        J = np.eye(T)[::-1]
        Rinv = np.linalg.inv(A)
        c = (1.0 / T) / max(Rinv.max(), 1e-12)
        assert np.abs(L - np.sqrt(c) * J @ np.linalg.inv(Lb.T) @ J).max() < 1e-9 * max(np.abs(L).max(), 1.0)
        s = (1.0 / T) / np.maximum(Rinv.max(0), 1e-12)
        x = np.random.default_rng(T).normal(size=T)
        assert np.abs(M @ x - np.linalg.solve(A, s * x)).max() < 1e-9 * max(np.abs(M @ x).max(), 1.0)
        assert np.array_equal(R, R[::-1, ::-1])   # persymmetric: J R J = R
