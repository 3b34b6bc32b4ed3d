"""GPU parity of the batched propagation (C ABI mqct_propagate_batch) against
the FP64 oracle, on the reference's H2O+H2 example (SYS_TYPE 8, the golden
matrix) and on an AT-MQCT case with a given classical path.

Tolerances: FP64 arithmetic -- channel probabilities within 1e-8 absolute and
identical step counts (same RK4 discretisation, summation order differs);
FP32 arithmetic -- probabilities within 2e-4 absolute and inelastic cross
sections within 1e-3 relative of the oracle."""
import os

import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g3(mq, oracle):
    g = np.load(os.path.join(GOLD, "g3_h2o_h2_type8.npz"))
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    tab = mq.PropagationTables.from_system(s, g["R"], g["mat"], float(g["mass_red"]))
    assert tab.P == 591
    otab = oracle.OracleTables(tab.j12, tab.m12, tab.ej, tab.ind_mat, tab.R, tab.mat, tab.y2,
                               tab.mass_au)
    trajs, meta = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), float(g["mass_red"]), 1,
                                    float(g["time_step"]), float(g["rmax"]),
                                    time_lim=float(g["time_lim"]))
    return dict(g=g, s=s, tab=tab, otab=otab, trajs=trajs, meta=meta)


def _oracle_run(oracle, otab, trajs):
    ot = [oracle.make_traj(t.e_coll, t.l_real, t.s_st, t.dt, t.r_start, t.r_fin,
                           t.numb_orb_prds, t.numb_oscl_prds, t.time_lim, t.max_steps) for t in trajs]
    return oracle.propagate_batch(otab, ot)


def test_fp64_matches_oracle(mq, oracle, gpu_available, g3):
    sub = g3["trajs"][::11]
    amp, cls, diag = mq.propagate(g3["tab"], sub, arith=mq.PROP_FP64)
    oamp, ocls, odiag = _oracle_run(oracle, g3["otab"], sub)
    pg = mq.channel_probabilities(amp, g3["s"].indx_chann, 10)
    po_ = mq.channel_probabilities(oamp, g3["s"].indx_chann, 10)
    assert np.max(np.abs(pg - po_)) < 1e-8
    assert np.array_equal(diag[:, 1], odiag[:, 1])          # step counts
    assert np.allclose(diag[:, 0], odiag[:, 0], rtol=1e-14)  # finish times
    assert np.allclose(cls[:, :2], ocls[:, :2], rtol=1e-9, atol=1e-9)
    assert np.allclose(cls[:, 4:], ocls[:, 4:], rtol=1e-8, atol=1e-9)
    assert np.all(diag[:, 4] == 0)
    assert np.max(diag[:, 3]) < 1e-9                        # energy conservation (Hartree)


def test_fp32_cross_sections_match_oracle_and_reference(mq, oracle, gpu_available, g3):
    trajs = g3["trajs"]
    amp, cls, diag = mq.propagate(g3["tab"], trajs, arith=mq.PROP_FP32)
    oamp, ocls, odiag = _oracle_run(oracle, g3["otab"], trajs)
    idx = g3["s"].indx_chann
    pg = mq.channel_probabilities(amp, idx, 10)
    po_ = mq.channel_probabilities(oamp, idx, 10)
    assert np.max(np.abs(pg - po_)) < 2e-4
    m = g3["meta"]
    sg = mq.cross_sections(pg, 0, m["J_down"], m["J_up"], m["L_min"], m["k"])
    so = mq.cross_sections(po_, 0, m["J_down"], m["J_up"], m["L_min"], m["k"])
    assert np.allclose(sg[1:4], so[1:4], rtol=1e-3)
    ref = g3["g"]["sigma_U"]
    assert np.allclose(sg[1:4], ref[1:4], rtol=1e-3)
    assert np.allclose(np.abs(diag[:, 2]), 0, atol=1e-5)  # norm


def test_queue_refill_order_independent(mq, gpu_available, g3):
    """More trajectories than resident slots: results do not depend on position."""
    trajs = g3["trajs"][:6]
    a1, _, _ = mq.propagate(g3["tab"], trajs, arith=mq.PROP_FP64)
    a2, _, _ = mq.propagate(g3["tab"], trajs[::-1], arith=mq.PROP_FP64)
    assert np.array_equal(a1, a2[::-1])


def test_step_cap_sets_status(mq, gpu_available, g3):
    t = g3["trajs"][0]
    t.max_steps = 50
    amp, cls, diag = mq.propagate(g3["tab"], [t], arith=mq.PROP_FP32)
    assert diag[0, 4] == 1 and diag[0, 1] == 50


def _straight_path(b, v, R0, mass, n=4000):
    """Classical straight-line path records (t, R, P_R, theta, P_theta, phi, P_phi, pot)."""
    x0 = -np.sqrt(R0 ** 2 - b ** 2)
    tmax = 2 * abs(x0) / v
    t = np.linspace(0.0, tmax, n)
    x = x0 + v * t
    R = np.sqrt(x ** 2 + b ** 2)
    L = mass * v * b
    rec = np.zeros((n, 8))
    rec[:, 0] = t
    rec[:, 1] = R
    rec[:, 2] = mass * v * x / R
    rec[:, 3] = np.pi / 2
    rec[:, 5] = np.arctan2(b, x) - np.arctan2(b, x0)
    rec[:, 6] = L
    return rec


def test_at_mode_matches_oracle(mq, oracle, gpu_available):
    c1 = syn.config_c1()
    s = mq.CollisionSystem(1, c1["channels"][:6], BE=c1["BE"])
    R = mq.r_grid(120, 3.0, 20.0)
    mat, y2, sk = mq.build_matrix(s, R, c1["grid"], c1["pes"], precision=mq.PREC_FP64)
    tab = mq.PropagationTables.from_system(s, R, mat, c1["mass_amu"])
    otab = oracle.OracleTables(tab.j12, tab.m12, tab.ej, tab.ind_mat, tab.R, tab.mat, tab.y2,
                               tab.mass_au)
    mass = tab.mass_au
    E = 500.0 * syn.CM_TO_HARTREE
    v = np.sqrt(2 * E / mass)
    paths = [_straight_path(b, v, 20.0, mass) for b in (4.0, 6.0, 9.0)]
    trajs = [mq.Trajectory(E, 0.0, 1, 20.0, 20.0, 20.0) for _ in paths]
    amp, cls, diag = mq.propagate(tab, trajs, arith=mq.PROP_FP64, mode=mq.MODE_AT, at_paths=paths)
    for i, p in enumerate(paths):
        oamp, odiag = oracle.dotraject_at(otab, oracle.make_traj(E, 0.0, 1, 20.0, 20.0, 20.0), p)
        assert np.max(np.abs(amp[i] - oamp)) < 1e-9
        assert diag[i, 1] == odiag[1]
        assert abs(diag[i, 0] - odiag[0]) < 1e-9 * odiag[0]
    assert np.all(np.abs(diag[:, 2]) < 1e-8)
    # the path passes the coupling region: population leaves the initial state
    p = mq.channel_probabilities(amp, s.indx_chann, s.n_channels)
    assert p[0, 0] < 0.999
