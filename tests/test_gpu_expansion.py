"""GPU parity of the PES-expansion matrix build (SYS_TYPE 8): the reference's own
H2O + H2 matrix (MTRX.DAT, built by the reference from PES_EXPAN_TERMS.DAT) is
reproduced from the same expansion terms, up to the per-level eigenvector phase
(see tests/test_oracle_expansion.py), and the GPU agrees with the oracle."""
import os

import numpy as np
import pytest

from test_oracle_expansion import level_gauge

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_expansion_matrix_matches_reference_and_oracle(mq, oracle, gpu_available):
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    g5 = np.load(os.path.join(GOLD, "g5_h2o_h2_expansion_terms.npz"))
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    m, y2, sk = mq.build_matrix_expansion(s, g5["R"], g5["labels"], g5["terms"], mij_cutoff=0.0)
    ref = g["mat"]
    gauge = level_gauge(s, m, ref)
    assert np.max(np.abs(m - gauge[:, None] * ref)) <= 1e-10 * np.abs(ref).max()
    ch = s.channels
    osys = oracle.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch,
                               vec1=s.vec1.reshape(-1), ldv=s.ldv)
    mo = oracle.expansion_matrix_type8(osys, osys.states(), s.ind_mat, g5["labels"], g5["terms"])
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()
    # spline of the columns: the host restatement of the reference's spline
    y2ref = mq.spline_y2(g5["R"], m)
    assert np.max(np.abs(y2 - y2ref)) <= 1e-10 * np.abs(y2ref).max()
    assert not sk.any()


def test_expansion_rejects_bad_terms(mq, gpu_available):
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    R = g["R"]
    with pytest.raises(mq.MqctError):
        mq.build_matrix_expansion(s, R, np.array([[1, 2, 0, 1]]), np.zeros((len(R), 1)))


def test_type7_expansion_matches_reference_and_oracle(mq, oracle, gpu_available):
    g = np.load(os.path.join(GOLD, "g5b_nd3_d2_type7.npz"))
    s = mq.CollisionSystem(7, g["channels"], A=float(g["A"]), C=float(g["C"]), BE=float(g["BE"]))
    m, y2, sk = mq.build_matrix_expansion(s, g["R"], g["labels"], g["terms"], e_unit="CM-1",
                                          mij_cutoff=0.0)
    ref = g["mat"]
    assert np.max(np.abs(m - ref)) <= 1e-11 * np.abs(ref).max()
    ch = s.channels
    osys = oracle.OracleSystem(7, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch, ldv=1)
    mo = oracle.expansion_matrix_type7(osys, osys.states(), s.ind_mat, g["labels"], g["terms"],
                                       mq.E_UNIT["CM-1"])
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()
    assert not sk.any()


def test_expansion_mij_cutoff_flags(mq, oracle, gpu_available):
    """MIJ_CUTOFF on the expansion path: elements whose |M| at the R points nearest
    r_cut1 and r_cut2 stays below the cut are zeroed and flagged, as in the
    direct-integration build."""
    g = np.load(os.path.join(GOLD, "g5b_nd3_d2_type7.npz"))
    s = mq.CollisionSystem(7, g["channels"], A=float(g["A"]), C=float(g["C"]), BE=float(g["BE"]))
    R = g["R"]
    m0, _, _ = mq.build_matrix_expansion(s, R, g["labels"], g["terms"], mij_cutoff=0.0)
    cut_cm = 5.0   # 220 symmetry zeros and 46 small elements fall below it
    m, y2, sk = mq.build_matrix_expansion(s, R, g["labels"], g["terms"], mij_cutoff=cut_cm)
    ir1, ir2 = np.argmin(np.abs(R - 6.0)), np.argmin(np.abs(R - 8.0))
    expect = np.maximum(np.abs(m0[:, ir1]), np.abs(m0[:, ir2])) < cut_cm * mq.CM_TO_HARTREE
    assert (expect & (np.abs(m0).max(axis=1) > 1e-12)).sum() > 20 and not expect.all()
    assert np.array_equal(sk.astype(bool), expect)
    assert np.all(m[expect] == 0.0) and np.array_equal(m[~expect], m0[~expect])


def test_expansion_plan_reuse(mq, gpu_available):
    """The plan forms the angular coefficients once: execute() with the example's terms
    equals the one-shot build, and with the terms doubled gives exactly twice the
    matrix and its spline (both linear in the terms; cut-off off)."""
    import torch
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    g5 = np.load(os.path.join(GOLD, "g5_h2o_h2_expansion_terms.npz"))
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    R, lab, T = g5["R"], g5["labels"], g5["terms"]
    m1, y1, _ = mq.build_matrix_expansion(s, R, lab, T, mij_cutoff=0.0)
    plan = mq.ExpansionPlan(s, R, lab, mij_cutoff=0.0)
    dT = torch.from_numpy(np.ascontiguousarray(T.T)).cuda()      # terms[t * nR + iR]
    dm = torch.empty((s.P, len(R)), dtype=torch.float64, device="cuda")
    dy = torch.empty_like(dm)
    dk = torch.empty(s.P, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # the plan runs on its own stream
    plan.execute(dT, dm, dy, dk)
    plan.sync()
    assert np.array_equal(dm.cpu().numpy(), m1) and np.array_equal(dy.cpu().numpy(), y1)
    dT2 = 2.0 * dT
    torch.cuda.synchronize()
    plan.execute(dT2, dm, dy, dk)
    plan.sync()
    assert np.array_equal(dm.cpu().numpy(), 2.0 * m1) and np.array_equal(dy.cpu().numpy(), 2.0 * y1)
    ang, ex = plan.timing()
    assert ang > 0.0 and ex > 0.0
    plan.close()


def test_expansion_high_j_direct_path(mq, oracle, gpu_available):
    """j = 20 rotor levels with an l1 = 20 term: the Clebsch-Gordan table of the angular
    set-up would exceed its size cap, so the coefficients are evaluated directly; the
    result agrees with the oracle as on the table path."""
    chans = [(20, 0, 20, 0), (19, 0, 19, 0), (20, 1, 20, 0)]
    s = mq.CollisionSystem(8, chans, A=27.88, B=9.28, C=14.52, BE=60.85)
    R = np.linspace(4.0, 12.0, 9)
    labels = np.array([[20, 0, 0, 20], [2, 0, 0, 2], [19, 2, 0, 19]], np.int32)
    rng = np.random.default_rng(3)
    terms = rng.standard_normal((len(R), len(labels)))
    m, _, _ = mq.build_matrix_expansion(s, R, labels, terms, mij_cutoff=0.0)
    ch = s.channels
    osys = oracle.OracleSystem(8, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], e_ch=s.e_ch,
                               vec1=s.vec1.reshape(-1), ldv=s.ldv)
    mo = oracle.expansion_matrix_type8(osys, osys.states(), s.ind_mat, labels, terms)
    assert np.abs(mo).max() > 0
    # at j = 20 the alternating Racah sums of the coefficients cancel several digits, and
    # the two evaluations (log-factorial exponentials here, the oracle's 3j routine there)
    # lose different ones: 6e-12 of the largest element
    assert np.max(np.abs(m - mo)) <= 1e-10 * np.abs(mo).max()


def test_identical_expansion_matches_reference_and_oracle(mq, oracle, gpu_available):
    from test_oracle_expansion import identical_gauge
    g = np.load(os.path.join(GOLD, "g5c_h2o_h2o_identical.npz"))
    s = mq.CollisionSystem(0, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           identical=True)
    m, y2, sk = mq.build_matrix_expansion(s, g["R"], g["labels"], g["terms"], e_unit="KCAL",
                                          mij_cutoff=0.0)
    gauge, err = identical_gauge(s, m, g["mat"])
    assert err <= 1e-10
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    mo = oracle.expansion_matrix_type0_identical(osys, (s.indx_chann, s.j12, s.m12, None),
                                                s.parity, s.ind_mat,
                                                 g["labels"], g["terms"], mq.E_UNIT["KCAL"])
    assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()
    # the term-list rule of identical partners (l1 >= l2) is enforced
    with pytest.raises(mq.MqctError):
        mq.build_matrix_expansion(s, g["R"], [[0, 0, 1, 0, 1]], np.zeros((2, 1)), e_unit="KCAL")
