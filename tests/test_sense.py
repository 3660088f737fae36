"""CG-SENSE restatement (CPU): pins the oracle's penalty against an explicit
pair-sum construction of Reg1's C'C, its SENSE operator pair against the
adjoint identity, and its qpwls_pcg1 iterates against the normal equations."""
import numpy as np

from mirt_b200 import workloads as wl
from oracle.sense_ref import Sense64, qpwls_pcg1


def _problem(seed=0, N=16, K=32, C=3):
    rng = np.random.default_rng(seed)
    om = wl.ga_radial(20, 2 * N)
    sens = wl.coil_maps((N, N), C, rng).transpose(1, 0, 2)   # [N2, N1, C]
    A = Sense64(om, N, K, sens, beta=0.5)
    return A, rng


def test_reg1_matches_pair_sums():
    A, _ = _problem()
    N = A.N
    M = np.zeros((N * N, N * N))
    for i in range(N * N):
        e = np.zeros(N * N)
        e[i] = 1
        M[:, i] = A.reg(e.reshape(N, N)).real.ravel()
    M2 = np.zeros_like(M)
    for i2 in range(N):
        for i1 in range(N):
            for d1, d2, w in ((1, 0, 1), (0, 1, 1), (1, 1, 2 ** -.5), (-1, 1, 2 ** -.5)):
                j1, j2 = i1 - d1, i2 - d2
                if 0 <= j1 < N and 0 <= j2 < N:
                    a, b = i2 * N + i1, j2 * N + j1
                    M2[a, a] += w
                    M2[b, b] += w
                    M2[a, b] -= w
                    M2[b, a] -= w
    assert np.abs(M - 0.5 * M2).max() < 1e-12


def test_sense_pair_is_adjoint():
    A, rng = _problem(1)
    x = rng.standard_normal((A.N, A.N)) + 1j * rng.standard_normal((A.N, A.N))
    y = rng.standard_normal((A.st["M"], A.C)) + 1j * rng.standard_normal((A.st["M"], A.C))
    lhs = np.vdot(A.forward(x), y)
    rhs = np.vdot(x, A.adjoint(y))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_pcg_iterates_solve_normal_equations():
    A, rng = _problem(2)
    xt = wl.ellipses(A.N, 4, rng).T
    y = A.forward(xt)
    xs = qpwls_pcg1(np.zeros_like(xt), A, None, y, 150)
    x = xs[-1]
    r = A.adjoint(y - A.forward(x)) - A.reg(x)
    b = A.adjoint(y)
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(b)
