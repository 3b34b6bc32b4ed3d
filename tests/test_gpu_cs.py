"""GPU parity of the coupled-states approximation (MQCT_MODE_CS): the reference's MF + He
CS example (fixture tests/golden/g4_type4_layout.npz, see tests/test_oracle_cs.py) run
through mqct_propagate_batch against the oracle and the reference's printed results,
in FP64 (probabilities within 1e-8 of the oracle, 2e-7 of the 8 printed digits) and
FP32 (2e-4), the plan switch, AT-MQCT with CS against the oracle (1e-9), and the elastic
scattering of ELAST_CALC (deflection function, phases, elastic cross section) from the
final classical states against the printed ones."""
import os

import numpy as np
import pytest

from test_oracle_cs import channel_prob, g4_tables, g4_trajs

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g4(mq, oracle):
    g = np.load(os.path.join(GOLD, "g4_type4_layout.npz"))
    s = mq.CollisionSystem(4, g["channels"], A=float(g["A"]), B=float(g["B"]), C=float(g["C"]))
    assert np.array_equal(s.indx_chann, g["states"][:, 1])
    tab = mq.PropagationTables.from_system(s, g["R"], g["mat"], float(g["mass_red"]))
    otab = g4_tables(oracle, g)
    otr, k, jmax = g4_trajs(oracle, g, True)
    trajs = [mq.Trajectory(t.e_coll, t.l_real, 1, t.dt, t.r_start, t.r_fin,
                           time_lim=float(g["time_lim"])) for t in otr]
    return dict(g=g, s=s, tab=tab, otab=otab, otr=otr, trajs=trajs, k=k, jmax=jmax)


def test_cs_fp64_matches_oracle_and_reference(mq, oracle, gpu_available, g4):
    amp, cls, diag = mq.propagate(g4["tab"], g4["trajs"], arith=mq.PROP_FP64,
                                  coupled_states=True)
    oamp, ocls, odiag = oracle.propagate_batch(g4["otab"], g4["otr"])
    pg = channel_prob(amp, g4["g"]["states"])
    po_ = channel_prob(oamp, g4["g"]["states"])
    assert np.max(np.abs(pg - po_)) < 1e-8
    assert np.array_equal(diag[:, 1], odiag[:, 1])
    r = g4["g"]["opacity"][:, 2:]
    assert np.max(np.abs(pg - r) / r) < 2e-7
    assert np.allclose(cls[:, 5], ocls[:, 5], rtol=1e-13)          # P_phi unchanged
    # states of other m12 than the initial state's keep exactly zero amplitude
    N = len(g4["g"]["states"])
    other = g4["g"]["states"][:, 3] != 0
    assert np.all(amp[:, :N][:, other] == 0) and np.all(amp[:, N:][:, other] == 0)
    sig = mq.cross_sections(pg, 0, 0, g4["jmax"], 0, g4["k"])
    assert np.allclose(sig[1:], g4["g"]["sigma_U"][1:], rtol=2e-7)


def test_cs_fp32_and_plan_switch(mq, oracle, gpu_available, g4):
    amp, _, _ = mq.propagate(g4["tab"], g4["trajs"], arith=mq.PROP_FP32, coupled_states=True)
    pg = channel_prob(amp, g4["g"]["states"])
    assert np.max(np.abs(pg - g4["g"]["opacity"][:, 2:])) < 2e-4
    plan = mq.PropagationPlan(g4["tab"], arith=mq.PROP_FP64)
    plan.set_coupled_states(True)
    a1, _, _ = plan.run(g4["trajs"][::5])
    ref, _, _ = mq.propagate(g4["tab"], g4["trajs"][::5], arith=mq.PROP_FP64,
                             coupled_states=True)
    assert np.array_equal(a1, ref)
    plan.set_coupled_states(False)
    a0, _, _ = plan.run(g4["trajs"][::5])
    full, _, _ = mq.propagate(g4["tab"], g4["trajs"][::5], arith=mq.PROP_FP64)
    assert np.array_equal(a0, full) and not np.array_equal(a0, a1)
    plan.close()


def test_cs_at_mode_matches_oracle(mq, oracle, gpu_available, g4):
    """AT-MQCT with CS: paths saved by a standard CS run of the oracle, then the
    amplitudes along them (DERIVS_BK_adia with the CS skips)."""
    idx = [3, 17, 30]
    paths = [oracle.dotraject_record(g4["otab"], g4["otr"][i])[3] for i in idx]
    trajs = [g4["trajs"][i] for i in idx]
    amp, _, diag = mq.propagate(g4["tab"], trajs, arith=mq.PROP_FP64, mode=mq.MODE_AT,
                                at_paths=paths, coupled_states=True)
    for n, i in enumerate(idx):
        oamp, odiag = oracle.dotraject_at(g4["otab"], g4["otr"][i], paths[n])
        assert np.max(np.abs(amp[n] - oamp)) < 1e-9
        assert diag[n, 1] == odiag[1]


def test_elastic_scattering_matches_reference(mq, gpu_available, g4):
    """ELAST_CALC from the propagation's final classical states: the deflection function
    (DEFLECTION_FUNCTION.out, 8 printed digits) within 1e-6 rad, the scattering phases
    within 1e-5 rad, and the elastic cross section of CROSS_SECTIONS.out within 1e-6
    relative."""
    amp, cls, diag = mq.propagate(g4["tab"], g4["trajs"], arith=mq.PROP_FP64,
                                  coupled_states=True)
    d = g4["g"]["deflection"]
    chi = mq.deflection_angles(cls, g4["trajs"], g4["tab"].mass_au)
    assert np.max(np.abs(chi - d[:, 2])) < 1e-6
    l = np.array([t.l_real for t in g4["trajs"]])
    ph = mq.scattering_phases(l, chi)
    assert np.max(np.abs(ph - d[:, 3])) < 1e-5
    pg = channel_prob(amp, g4["g"]["states"])
    sig = mq.elastic_cross_section(l, pg[:, 0], ph, g4["k"])
    assert abs(sig / g4["g"]["sigma_U"][0] - 1) < 1e-6
