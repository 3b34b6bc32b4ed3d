"""GPU parity of the CALC_EXPANSION_TERMS projection (SYS_TYPE 7, 8, 0) with the oracle
on seeded PES tables, the known-answer property on the GPU, and the device pipeline
projection -> expansion matrix against the oracle's direct quadrature.

Tolerance: |GPU - oracle| <= 1e-12 max|V| 16 pi^2 per term, 16 pi^2 being the measure of
the angular grid; both sum the same FP64 products in different orders."""
import os

import numpy as np
import pytest

from test_oracle_projection import CM, LAB0, LAB8, _basis

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _bound(V):
    return 1e-12 * np.abs(V).max() * 16 * np.pi ** 2


@pytest.mark.parametrize("sys_type,golden,shape,eq", [
    (8, "g5_h2o_h2_expansion_terms.npz", (10, 12, 10, 12), True),
    (8, "g5_h2o_h2_expansion_terms.npz", (9, 11, 10, 7), False),
    (7, "g5b_nd3_d2_type7.npz", (12, 10, 8, 12), True),
    (0, "g1_h2o_h2o_at.npz", (6, 8, 8, 6, 6), True),
    (0, "g5c_h2o_h2o_identical.npz", (6, 8, 7, 6, 5), False),
])
def test_projection_matches_oracle(mq, oracle, gpu_available, sys_type, golden, shape, eq):
    labels = np.load(os.path.join(GOLD, golden))["labels"]
    if len(labels) > 120:
        labels = labels[::4]
    nR = 4
    rng = np.random.default_rng(11)
    V = rng.normal(size=(nR,) + shape) * 1e3 + 50.0
    T, Ti = mq.project_terms(sys_type, labels, V, eq_gamma=eq,
                             identical=golden.startswith("g5c"))
    To, Tio = oracle.project_terms(sys_type, labels, V, eq_gamma=eq)
    assert T.shape == (nR, len(labels))
    assert np.max(np.abs(T - To.T)) <= _bound(V)
    assert np.max(np.abs(Ti - Tio.T)) <= _bound(V)


@pytest.mark.parametrize("sys_type,labels,shape", [(8, LAB8, (8, 14, 14, 8)),
                                                   (0, LAB0, (6, 14, 14, 6, 6))])
def test_projection_recovers_the_coefficients_on_gpu(mq, oracle, gpu_available, sys_type, labels,
                                                     shape):
    W = _basis(oracle, sys_type, labels, shape)
    v = np.random.default_rng(5).normal(size=(len(labels), 3)) * 100.0
    V = np.einsum("tr,t...->r...", v, W)
    T, Ti = mq.project_terms(sys_type, labels, V)
    assert np.max(np.abs(T.T - v)) <= 1e-11 * np.abs(v).max()
    assert np.max(np.abs(Ti)) <= 1e-11 * np.abs(v).max()


def test_device_pipeline_projection_to_matrix(mq, oracle, gpu_available):
    """V on the device -> terms on the device (ProjectionPlan) -> Mat_el on the device
    (ExpansionPlan); equals the oracle's direct quadrature of the same V (type 0)."""
    import torch

    g = np.load(os.path.join(GOLD, "g1_h2o_h2o_at.npz"))
    s = mq.CollisionSystem(0, g["channels"][:4], A=float(g["A"]), B=float(g["B"]),
                           C=float(g["C"]))
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    shape = (8, 14, 14, 8, 8)
    W = _basis(oracle, 0, LAB0, shape)
    R = np.array([5.0, 6.5, 8.0])
    v = np.random.default_rng(3).normal(size=(len(LAB0), len(R))) * 100.0
    V = np.einsum("tr,t...->r...", v, W)
    pp = mq.ProjectionPlan(0, LAB0, shape)
    dV = torch.from_numpy(V).cuda()
    dT = torch.empty((len(LAB0), len(R)), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    pp.execute(dV, len(R), dT)
    pp.sync()
    ep = mq.ExpansionPlan(s, R, LAB0, mij_cutoff=0.0)
    dm = torch.empty((s.P, len(R)), dtype=torch.float64, device="cuda")
    dk = torch.empty(s.P, dtype=torch.int32, device="cuda")
    ep.execute(dT, dm, 0, dk, e_unit="CM-1")
    ep.sync()
    n2, n3, n4, n5, n6 = shape
    pes = oracle.OraclePes(0, 0, np.zeros(1), table=V.reshape(-1))
    direct, _, _ = oracle.build_matrix(osys, osys.states(), s.ind_mat, R,
                                       (n3, n5, 0, n4, n2, n6, 1), pes, mij_cut=0.0)
    m = dm.cpu().numpy()
    assert np.max(np.abs(m - direct)) <= 1e-10 * np.abs(direct).max()
    assert np.allclose(dT.cpu().numpy(), v, rtol=0, atol=1e-11 * np.abs(v).max())
    ga, al, te = pp.timing()
    assert ga > 0 and al > 0 and te > 0
    pp.close()
    ep.close()


def test_projection_plan_reuse(mq, gpu_available):
    import torch

    labels = np.load(os.path.join(GOLD, "g5_h2o_h2_expansion_terms.npz"))["labels"]
    shape = (8, 10, 8, 10)
    rng = np.random.default_rng(2)
    V = rng.normal(size=(6,) + shape)
    T1, I1 = mq.project_terms(8, labels, V)
    pp = mq.ProjectionPlan(8, labels, shape)
    dV = torch.from_numpy(V).cuda()
    dT = torch.empty((len(labels), 6), dtype=torch.float64, device="cuda")
    dI = torch.empty_like(dT)
    torch.cuda.synchronize()
    pp.execute(dV, 6, dT, dI)
    pp.sync()
    assert np.array_equal(dT.cpu().numpy(), T1.T) and np.array_equal(dI.cpu().numpy(), I1.T)
    # fewer R points, then the scaled table: the same sums, in the same order
    dT2 = torch.empty((len(labels), 2), dtype=torch.float64, device="cuda")
    dV2 = (2.0 * dV[:2]).contiguous()
    torch.cuda.synchronize()
    pp.execute(dV2, 2, dT2)
    pp.sync()
    assert np.array_equal(dT2.cpu().numpy(), 2.0 * T1[:2].T)
    pp.close()


def test_projection_many_pairs_and_long_gamma_rows(mq, oracle, gpu_available):
    """Type 0 with 41 (nju1, nju2) pairs (three register passes of the gamma contraction)
    and n_gamma1 x n_gamma2 = 72 points per row (two staged chunks)."""
    labels = [(4, n1, 4, n2, 4) for n1 in range(5) for n2 in range(-4, 5) if n1 > 0 or n2 >= 0]
    assert len(labels) == 41
    V = np.random.default_rng(4).normal(size=(2, 4, 6, 5, 9, 8)) * 300.0
    T, Ti = mq.project_terms(0, labels, V, eq_gamma=False)
    To, Tio = oracle.project_terms(0, labels, V, eq_gamma=False)
    assert np.max(np.abs(T - To.T)) <= _bound(V)
    assert np.max(np.abs(Ti - Tio.T)) <= _bound(V)
