"""GPU parity of the lockstep propagation engine (MQCT_ENGINE_LOCKSTEP: all trajectories
of a batch advance one RK4 stage per round, grouped by spline interval) against the oracle
and against the per-trajectory kernel, on the reference's H2O + H2 example (SYS_TYPE 8,
the golden matrix: 104 states, 11 m-blocks) and on the 969-state asymmetric-top system
(17 m-blocks of up to 81 states) with trajectories of the propagation benchmark.

Tolerances: FP64 arithmetic -- probabilities within 1e-8 absolute of the oracle, identical
step counts and finish times (the same RK4 discretisation; the spline applied as four knot
products, another rounding order) and within 1e-10 of the per-trajectory FP64 kernel;
FP32 arithmetic -- probabilities within 2e-4 of the oracle and cross sections within 1e-3
relative of the oracle and of the reference's printed ones, as for the per-trajectory
kernel."""
import numpy as np
import pytest

from test_gpu_propagate import _oracle_run, g3  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


def _run(mq, tab, trajs, arith, engine):
    plan = mq.PropagationPlan(tab, arith=arith)
    plan.set_engine(engine)
    amp, cls, diag = plan.run(trajs)
    eng = plan.engine()
    plan.close()
    return amp, cls, diag, eng


def test_fp64_matches_oracle_and_per_trajectory_kernel(mq, oracle, gpu_available, g3):
    sub = g3["trajs"][::11]
    amp, cls, diag, eng = _run(mq, g3["tab"], sub, mq.PROP_FP64, mq.ENGINE_LOCKSTEP)
    assert eng[0] == mq.ENGINE_LOCKSTEP and eng[1] > 0
    oamp, ocls, odiag = _oracle_run(oracle, g3["otab"], sub)
    idx = g3["s"].indx_chann
    pg = mq.channel_probabilities(amp, idx, 10)
    po_ = mq.channel_probabilities(oamp, idx, 10)
    assert np.max(np.abs(pg - po_)) < 1e-8
    assert np.array_equal(diag[:, 1], odiag[:, 1])          # step counts
    assert np.allclose(diag[:, 0], odiag[:, 0], rtol=1e-14)  # finish times
    assert np.allclose(cls[:, :2], ocls[:, :2], rtol=1e-9, atol=1e-9)
    assert np.all(diag[:, 4] == 0)
    assert np.max(diag[:, 3]) < 1e-9                        # energy conservation (Hartree)
    a2, c2, d2, e2 = _run(mq, g3["tab"], sub, mq.PROP_FP64, mq.ENGINE_PER_TRAJECTORY)
    assert e2[0] == mq.ENGINE_PER_TRAJECTORY
    assert np.max(np.abs(amp - a2)) < 1e-10
    assert np.array_equal(diag[:, [1, 4, 5, 6]], d2[:, [1, 4, 5, 6]])
    assert np.allclose(diag[:, 7], d2[:, 7], rtol=1e-9, atol=1e-14)


def test_fp32_cross_sections_match_oracle_and_reference(mq, oracle, gpu_available, g3):
    trajs = g3["trajs"]
    amp, cls, diag, eng = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_LOCKSTEP)
    assert eng[0] == mq.ENGINE_LOCKSTEP
    oamp, ocls, odiag = _oracle_run(oracle, g3["otab"], trajs)
    idx = g3["s"].indx_chann
    pg = mq.channel_probabilities(amp, idx, 10)
    po_ = mq.channel_probabilities(oamp, idx, 10)
    assert np.max(np.abs(pg - po_)) < 2e-4
    m = g3["meta"]
    sg = mq.cross_sections(pg, 0, m["J_down"], m["J_up"], m["L_min"], m["k"])
    so = mq.cross_sections(po_, 0, m["J_down"], m["J_up"], m["L_min"], m["k"])
    assert np.allclose(sg[1:4], so[1:4], rtol=1e-3)
    assert np.allclose(sg[1:4], g3["g"]["sigma_U"][1:4], rtol=1e-3)
    assert np.allclose(np.abs(diag[:, 2]), 0, atol=1e-5)  # norm


def test_stop_rules_and_skipped_trajectories(mq, gpu_available, g3):
    """Step caps (status 1), time limits, an impact parameter beyond RMAX (status 2, not
    propagated, the initial unit vector returned) and finished ones in one batch: the same
    diagnostics as the per-trajectory kernel."""
    base = g3["trajs"]
    t0 = base[5]
    trajs = [base[3], base[40], base[90]]
    trajs.append(mq.Trajectory(t0.e_coll, t0.l_real, 1, t0.dt, t0.r_start, t0.r_fin,
                               max_steps=37))
    trajs.append(mq.Trajectory(t0.e_coll, 1e5, 2, t0.dt, t0.r_start, t0.r_fin, max_steps=100))
    trajs.append(mq.Trajectory(t0.e_coll, t0.l_real, 3, t0.dt, t0.r_start, t0.r_fin,
                               time_lim=t0.dt * 50.5, max_steps=0))
    amp, cls, diag, eng = _run(mq, g3["tab"], trajs, mq.PROP_FP64, mq.ENGINE_LOCKSTEP)
    a2, c2, d2, _ = _run(mq, g3["tab"], trajs, mq.PROP_FP64, mq.ENGINE_PER_TRAJECTORY)
    assert eng[0] == mq.ENGINE_LOCKSTEP
    assert list(diag[:, 4]) == [0, 0, 0, 1, 2, 0]
    assert diag[3, 1] == 37 and diag[5, 1] == 51
    assert np.array_equal(diag[:, [0, 1, 4, 5, 6]], d2[:, [0, 1, 4, 5, 6]])
    assert np.max(np.abs(amp - a2)) < 1e-10
    assert np.allclose(cls, c2, rtol=1e-9, atol=1e-9)
    N = g3["tab"].n_states
    unit = np.zeros(2 * N)
    unit[1] = 1.0
    assert np.array_equal(amp[4], unit) and np.array_equal(a2[4], unit)


def test_engine_choice_and_device_buffers(mq, gpu_available, g3):
    """MQCT_ENGINE_AUTO keeps small batches on the per-trajectory kernel; the lockstep
    engine through mqct_prop_plan_run_device gives the host-buffer results."""
    import torch
    trajs = g3["trajs"][:12]
    plan = mq.PropagationPlan(g3["tab"], arith=mq.PROP_FP64)
    amp0, cls0, diag0 = plan.run(trajs)
    assert plan.engine()[0] == mq.ENGINE_PER_TRAJECTORY
    plan.set_engine(mq.ENGINE_LOCKSTEP)
    amp1, cls1, diag1 = plan.run(trajs)
    assert plan.engine()[0] == mq.ENGINE_LOCKSTEP
    arr = mq._traj_array(trajs)
    raw = np.frombuffer(bytes(arr), dtype=np.uint8)
    d_init = torch.from_numpy(raw.copy()).cuda()
    N, n = g3["tab"].n_states, len(trajs)
    d_amp = torch.zeros(n * 2 * N, dtype=torch.float64, device="cuda")
    d_cls = torch.zeros(n * 6, dtype=torch.float64, device="cuda")
    d_diag = torch.zeros(n * 8, dtype=torch.float64, device="cuda")
    plan.run_device(d_init.data_ptr(), n, d_amp.data_ptr(), d_cls.data_ptr(), d_diag.data_ptr())
    plan.sync()
    assert plan.engine()[0] == mq.ENGINE_LOCKSTEP
    assert np.array_equal(d_amp.cpu().numpy().reshape(n, 2 * N), amp1)
    assert np.array_equal(d_diag.cpu().numpy().reshape(n, 8), diag1)
    assert np.max(np.abs(amp1 - amp0)) < 1e-10
    with pytest.raises(mq.MqctError):
        plan.set_engine(7)
    plan.close()


@pytest.fixture(scope="module")
def c2_tables(mq, gpu_available):
    """The 969-state asymmetric top + atom matrix (2-D reference grid) and 192 trajectories
    of the propagation benchmark's set (b ~ U(0, 15) bohr, E log-uniform 50-2000 cm^-1)."""
    from mqct_b200 import synthetic as syn
    c2 = syn.config_c2(alpha_grid=False)
    s = mq.CollisionSystem(4, c2["channels"], A=c2["A"], B=c2["B"], C=c2["C"])
    R = mq.r_grid(c2["nR"], c2["rmin"], c2["rmax"])
    mat = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=mq.PREC_FP64)[0]
    tab = mq.PropagationTables.from_system(s, R, mat, c2["mass_amu"])
    c3 = syn.config_c3()
    n = 192
    E = c3["E_cm"][:n] * syn.CM_TO_HARTREE
    k = np.sqrt(2 * tab.mass_au * E)
    l = np.sqrt((c3["b"][:n] * k) ** 2 + 0.25) - 0.5
    trajs = [mq.Trajectory(float(E[i]), float(l[i]), 1 + (i % 7), c3["dt"], c3["r_fin"],
                           c3["r_fin"], max_steps=400000) for i in range(n)]
    return dict(s=s, tab=tab, trajs=trajs)


def test_asym_top_system_matches_per_trajectory_kernel(mq, gpu_available, c2_tables):
    s, trajs = c2_tables["s"], c2_tables["trajs"]
    tab = c2_tables["tab"]
    a_ls, _, d_ls, eng = _run(mq, tab, trajs, mq.PROP_FP64, mq.ENGINE_LOCKSTEP)
    a_pt, _, d_pt, _ = _run(mq, tab, trajs, mq.PROP_FP64, mq.ENGINE_PER_TRAJECTORY)
    assert eng[0] == mq.ENGINE_LOCKSTEP
    assert np.array_equal(d_ls[:, 1], d_pt[:, 1])
    p_ls = mq.channel_probabilities(a_ls, s.indx_chann, s.n_channels)
    p_pt = mq.channel_probabilities(a_pt, s.indx_chann, s.n_channels)
    assert np.max(np.abs(p_ls - p_pt)) < 1e-9
    # the energy error of the RK4 discretisation, not of the engine
    assert np.allclose(d_ls[:, 3], d_pt[:, 3], rtol=1e-5, atol=1e-12)
    a32, _, d32, _ = _run(mq, tab, trajs, mq.PROP_FP32, mq.ENGINE_LOCKSTEP)
    p32 = mq.channel_probabilities(a32, s.indx_chann, s.n_channels)
    assert np.max(np.abs(p32 - p_pt)) < 2e-4
    assert np.all(d32[:, 4] == 0)


def test_lockstep_tail_on_resident_engine(mq, gpu_available, c2_tables):
    """MQCT_ENGINE_LOCKSTEP_TAIL (the plan's choice for large FP32 batches): the lockstep
    engine hands the trajectories still running to the resident engine at a graph boundary
    (here after the first graph: the batch is below the hand-over count), which continues
    each from the start of its RK4 step; the results are those of the FP32 per-trajectory
    kernel to FP32 rounding."""
    s, trajs, tab = c2_tables["s"], c2_tables["trajs"], c2_tables["tab"]
    plan = mq.PropagationPlan(tab, mq.PROP_FP32)
    plan.set_engine(mq.ENGINE_LOCKSTEP_TAIL)
    a_t, _, d_t = plan.run(trajs)
    eng, rounds = plan.engine()
    assert eng == mq.ENGINE_LOCKSTEP_TAIL and rounds > 0 and 0 < plan.handed() <= len(trajs)
    plan.close()
    a_p, _, d_p, _ = _run(mq, tab, trajs, mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY)
    p_t = mq.channel_probabilities(a_t, s.indx_chann, s.n_channels)
    p_p = mq.channel_probabilities(a_p, s.indx_chann, s.n_channels)
    assert np.max(np.abs(p_t - p_p)) < 5e-5
    assert np.all(d_t[:, 4] == 0)
    assert np.allclose(d_t[:, 1], d_p[:, 1], rtol=1e-3)
    # the norm errors are the RK4 discretisation's (long FP32 trajectories drift), the same
    # for both engines to rounding
    assert np.allclose(d_t[:, 2], d_p[:, 2], rtol=0.05, atol=1e-6)
