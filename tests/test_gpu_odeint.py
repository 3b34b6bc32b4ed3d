"""GPU parity of the adaptive integrator (PROPAGATOR = ODEINT) against the oracle's
restatement of the reference's scheme: standard MQCT on the reference's H2O + H2
matrix (G3) and AT-MQCT on its H2O + H2O second run (G1).

The minimum step is positive (1 a.u. here, 20 a.u. for the AT paths): the
reference's error scale |y| + |h dy/dt| + 1e-30 asks for relative accuracy eps even
on amplitudes at rounding level (~1e-23 in this system), so with hmin = 0 the step
collapses wherever rounding noise dominates them -- on the CPU and the GPU alike,
but at places that depend on the rounding.  With hmin > 0 such steps are taken at
hmin, the results do not depend on where that happens (1e-14 between hmin = 0 and
hmin = 1 a.u. in the oracle), and the cost stays bounded.

Tolerances: probabilities within 1e-8 absolute, identical outer step counts and
finish times.  ODEINT runs in FP64 arithmetic only."""
import numpy as np
import pytest

from test_oracle_g1 import AMU as AMU1, KCAL, _g1
from test_oracle_golden import _g3

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g3(mq, oracle, gpu_available):
    g = _g3()
    s = mq.CollisionSystem(8, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]),
                           BE=float(g["BE"]))
    tab = mq.PropagationTables.from_system(s, g["R"], g["mat"], float(g["mass_red"]))
    otab = oracle.OracleTables(tab.j12, tab.m12, tab.ej, tab.ind_mat, tab.R, tab.mat, tab.y2,
                               tab.mass_au)
    trajs, meta = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), float(g["mass_red"]), 1,
                                    float(g["time_step"]), float(g["rmax"]),
                                    time_lim=float(g["time_lim"]))
    return dict(g=g, s=s, tab=tab, otab=otab, trajs=[trajs[l] for l in (40, 80, 110)])


def _oracle_trajs(oracle, trajs, eps, hmin):
    return [oracle.make_traj(t.e_coll, t.l_real, t.s_st, t.dt, t.r_start, t.r_fin,
                             t.numb_orb_prds, t.numb_oscl_prds, t.time_lim, t.max_steps,
                             method=1, eps=eps, hmin=hmin) for t in trajs]


def test_standard_mode_matches_oracle(mq, oracle, g3):
    integ = ("ODEINT", 1e-5, 1.0)
    amp, cls, diag = mq.propagate(g3["tab"], g3["trajs"], arith=mq.PROP_FP64, integrator=integ)
    oamp, ocls, odiag = oracle.propagate_batch(g3["otab"], _oracle_trajs(oracle, g3["trajs"], 1e-5, 1.0))
    pg = mq.channel_probabilities(amp, g3["s"].indx_chann, 10)
    po_ = mq.channel_probabilities(oamp, g3["s"].indx_chann, 10)
    assert np.max(np.abs(pg - po_)) < 1e-8
    assert np.array_equal(diag[:, 1], odiag[:, 1])
    assert np.allclose(diag[:, 0], odiag[:, 0], rtol=1e-14)
    assert np.allclose(cls[:, :2], ocls[:, :2], rtol=1e-8, atol=1e-8)
    assert np.all(diag[:, 4] == 0)
    # and the RK4 outputs the reference printed for these trajectories
    ref = g3["g"]["opacity"][[40, 80, 110], 2:]
    assert np.max(np.abs(pg - ref)) < 1e-6


def test_fp32_arithmetic_is_rejected(mq, g3):
    """ODEINT resolves every amplitude to relative eps, below FP32 rounding of the
    right-hand side: the library refuses the combination instead of collapsing steps."""
    with pytest.raises(mq.MqctError, match="FP64"):
        mq.propagate(g3["tab"], g3["trajs"], arith=mq.PROP_FP32, integrator=("ODEINT", 1e-5, 1.0))
    plan = mq.PropagationPlan(g3["tab"], arith=mq.PROP_FP32)
    with pytest.raises(mq.MqctError):
        plan.set_integrator(("ODEINT", 1e-5, 1.0))
    plan.close()


def test_plan_integrator_switch(mq, g3):
    """A plan switched to ODEINT and back to RK4 gives the one-shot results of each."""
    plan = mq.PropagationPlan(g3["tab"], arith=mq.PROP_FP64)
    r4 = plan.run(g3["trajs"])[0]
    plan.set_integrator(("ODEINT", 1e-5, 1.0))
    ro = plan.run(g3["trajs"])[0]
    plan.set_integrator(None)
    r4b = plan.run(g3["trajs"])[0]
    plan.close()
    a4 = mq.propagate(g3["tab"], g3["trajs"], arith=mq.PROP_FP64)[0]
    ao = mq.propagate(g3["tab"], g3["trajs"], arith=mq.PROP_FP64, integrator=("ODEINT", 1e-5, 1.0))[0]
    assert np.array_equal(r4, a4) and np.array_equal(r4b, a4) and np.array_equal(ro, ao)
    with pytest.raises(mq.MqctError):
        mq.propagate(g3["tab"], g3["trajs"], integrator=("ODEINT", 0.0, 0.0))


def test_at_mode_matches_oracle(mq, oracle, gpu_available):
    g = _g1()
    A, B, Cc = float(g["A"]), float(g["B"]), float(g["C"])
    mass_amu = float(g["mass_red"])
    s1 = mq.CollisionSystem(0, g["channels"][:1], A=A, B=B, C=Cc)
    s9 = mq.CollisionSystem(0, g["channels"], A=A, B=B, C=Cc)
    m1 = mq.build_matrix_expansion(s1, g["R"], g["labels"], g["terms"], e_unit="KCAL",
                                   mij_cutoff=0.0)[0]
    m9 = mq.build_matrix_expansion(s9, g["R"], g["labels"], g["terms"], e_unit="KCAL",
                                   mij_cutoff=0.0)[0]
    tab1 = mq.PropagationTables.from_system(s1, g["R"], m1, mass_amu)
    tab9 = mq.PropagationTables.from_system(s9, g["R"], m9, mass_amu)
    idx = [list(g["l"]).index(l) for l in (9, 85, 199)]
    t1, meta = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), mass_amu, 1,
                                 float(g["time_step1"]), float(g["rmax"]), dl=int(g["dl"]),
                                 time_lim=float(g["time_lim"]))
    t1 = [t1[i] for i in idx]
    paths = mq.propagate_record(tab1, t1, arith=mq.PROP_FP64)[3]
    t2, _ = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), mass_amu, 1,
                              float(g["time_step2"]), float(g["rmax"]), dl=int(g["dl"]),
                              time_lim=float(g["time_lim"]))
    t2 = [t2[i] for i in idx]
    integ = ("ODEINT", 1e-6, 20.0)
    amp, _, diag = mq.propagate(tab9, t2, arith=mq.PROP_FP64, mode=mq.MODE_AT, at_paths=paths,
                                integrator=integ)
    otab = oracle.OracleTables(tab9.j12, tab9.m12, tab9.ej, tab9.ind_mat, tab9.R, tab9.mat,
                               tab9.y2, tab9.mass_au)
    N = s9.n_states
    for i, t in enumerate(_oracle_trajs(oracle, t2, 1e-6, 20.0)):
        oamp, odiag = oracle.dotraject_at(otab, t, paths[i])
        assert np.max(np.abs(amp[i] - oamp)) < 1e-8
        assert diag[i, 0] == odiag[0] == paths[i][-1, 0]
    prob = mq.channel_probabilities(amp, s9.indx_chann, 9)
    ref = g["opacity2"][idx, 2:]
    assert np.max(np.abs(prob[1:] - ref[1:])) < 1e-6     # l = 85, 199


def test_bk_int_matches_oracle(mq, oracle, g3):
    """ODEINT with bikram_int on the GPU (one adaptive call over [0, TIME_LIM] with the
    stop rules after every step) against the oracle's bk_int restatement: the same finish
    times, probabilities within 1e-8, and the reference's RK4 probabilities within 1e-6."""
    integ = ("BK_INT", 1e-4, 10.0)
    amp, cls, diag = mq.propagate(g3["tab"], g3["trajs"], arith=mq.PROP_FP64, integrator=integ)
    ot = [oracle.make_traj(t.e_coll, t.l_real, t.s_st, t.dt, t.r_start, t.r_fin,
                           t.numb_orb_prds, t.numb_oscl_prds, t.time_lim, t.max_steps,
                           method=3, eps=1e-4, hmin=10.0) for t in g3["trajs"]]
    oamp, ocls, odiag = oracle.propagate_batch(g3["otab"], ot)
    pg = mq.channel_probabilities(amp, g3["s"].indx_chann, 10)
    po_ = mq.channel_probabilities(oamp, g3["s"].indx_chann, 10)
    assert np.max(np.abs(pg - po_)) < 1e-8
    assert np.allclose(diag[:, 0], odiag[:, 0], rtol=1e-12)
    assert np.all(cls[:, 0] > float(g3["g"]["rmax"]))
    ref = g3["g"]["opacity"][[40, 80, 110], 2:]
    assert np.max(np.abs(pg - ref)) < 1e-6
