"""GPU parity of the cluster-resident propagation engine (MQCT_ENGINE_RESIDENT: one
thread-block cluster per trajectory, the m-blocks split between its CTAs, each holding its
blocks' knot rows in shared memory) against the oracle, the reference's printed cross
sections and the per-trajectory kernel, on the reference's H2O + H2 example (SYS_TYPE 8,
the golden matrix: 104 states, 11 m-blocks) and on the 969-state asymmetric-top system
(17 m-blocks of up to 81 states) with trajectories of the propagation benchmark.

Tolerances (FP32 arithmetic, as for the per-trajectory kernel): probabilities within 2e-4
of the oracle and of the FP64 per-trajectory kernel, cross sections within 1e-3 relative
of the oracle and of the reference's printed ones; within 5e-5 of the FP32 per-trajectory
kernel (the same products, other summation orders) and between cluster sizes."""
import numpy as np
import pytest

from test_gpu_lockstep import c2_tables  # noqa: F401  (fixture)
from test_gpu_propagate import _oracle_run, g3  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


def _run(mq, tab, trajs, arith, engine, cluster=0):
    plan = mq.PropagationPlan(tab, arith=arith)
    plan.set_engine(engine)
    plan.set_cluster(cluster)
    amp, cls, diag = plan.run(trajs)
    eng = plan.engine()[0]
    shape = plan.cluster()
    plan.close()
    return amp, cls, diag, eng, shape


def test_cross_sections_match_oracle_and_reference(mq, oracle, gpu_available, g3):
    trajs = g3["trajs"]
    amp, cls, diag, eng, shape = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_RESIDENT)
    assert eng == mq.ENGINE_RESIDENT and shape[0] >= 2 and shape[1] >= 1
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
    assert np.all(diag[:, 4] == 0)
    a2, c2, d2, e2, _ = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY)
    assert e2 == mq.ENGINE_PER_TRAJECTORY
    p2 = mq.channel_probabilities(a2, idx, 10)
    assert np.max(np.abs(pg - p2)) < 5e-5
    assert np.allclose(cls[:, 0], c2[:, 0], rtol=1e-4)


def test_stop_rules_and_skipped_trajectories(mq, gpu_available, g3):
    """Step caps (status 1), time limits, an impact parameter beyond RMAX (status 2, not
    propagated, the initial unit vector returned) and finished ones in one batch: the
    per-trajectory kernel's diagnostics."""
    base = g3["trajs"]
    t0 = base[5]
    trajs = [base[3], base[40], base[90]]
    trajs.append(mq.Trajectory(t0.e_coll, t0.l_real, 1, t0.dt, t0.r_start, t0.r_fin,
                               max_steps=37))
    trajs.append(mq.Trajectory(t0.e_coll, 1e5, 2, t0.dt, t0.r_start, t0.r_fin, max_steps=100))
    trajs.append(mq.Trajectory(t0.e_coll, t0.l_real, 3, t0.dt, t0.r_start, t0.r_fin,
                               time_lim=t0.dt * 50.5, max_steps=0))
    amp, cls, diag, eng, _ = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_RESIDENT)
    a2, c2, d2, _, _ = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY)
    assert eng == mq.ENGINE_RESIDENT
    assert list(diag[:, 4]) == [0, 0, 0, 1, 2, 0]
    assert diag[3, 1] == 37 and diag[5, 1] == 51
    assert np.array_equal(diag[3:, [0, 1, 4]], d2[3:, [0, 1, 4]])
    assert np.max(np.abs(amp - a2)) < 1e-4
    N = g3["tab"].n_states
    unit = np.zeros(2 * N)
    unit[1] = 1.0
    assert np.array_equal(amp[4], unit) and np.array_equal(a2[4], unit)
    assert np.array_equal(cls[4], c2[4]) and np.array_equal(diag[4], d2[4])


def test_engine_choice_cluster_sizes_and_device_buffers(mq, gpu_available, g3):
    """An FP64 plan does not take the resident engine (it reports no cluster); a small FP32
    batch takes it under MQCT_ENGINE_AUTO; the cluster size can be forced, with results
    equal to FP32 rounding; mqct_prop_plan_run_device gives the host-buffer results."""
    import torch
    trajs = g3["trajs"][:12]
    p64 = mq.PropagationPlan(g3["tab"], arith=mq.PROP_FP64)
    p64.set_engine(mq.ENGINE_RESIDENT)
    assert p64.cluster() == (0, 0)
    p64.run(trajs)
    assert p64.engine()[0] != mq.ENGINE_RESIDENT
    p64.close()
    plan = mq.PropagationPlan(g3["tab"], arith=mq.PROP_FP32)
    amp0, _, _ = plan.run(trajs)
    # MQCT_ENGINE_AUTO: a small FP32 batch takes the resident engine, on clusters of eight
    assert plan.engine()[0] == mq.ENGINE_RESIDENT and plan.cluster()[0] == 8
    plan.set_engine(mq.ENGINE_RESIDENT)
    plan.set_cluster(2)
    amp1, cls1, diag1 = plan.run(trajs)
    assert plan.engine()[0] == mq.ENGINE_RESIDENT and plan.cluster()[0] == 2
    plan.set_cluster(4)
    amp4, _, diag4 = plan.run(trajs)
    assert plan.engine()[0] == mq.ENGINE_RESIDENT and plan.cluster()[0] == 4
    p0 = mq.channel_probabilities(amp0, g3["s"].indx_chann, 10)
    p1 = mq.channel_probabilities(amp1, g3["s"].indx_chann, 10)
    p4 = mq.channel_probabilities(amp4, g3["s"].indx_chann, 10)
    assert np.max(np.abs(p1 - p4)) < 5e-5 and np.max(np.abs(p1 - p0)) < 5e-5
    plan.set_cluster(2)
    arr = mq._traj_array(trajs)
    raw = np.frombuffer(bytes(arr), dtype=np.uint8)
    d_init = torch.from_numpy(raw.copy()).cuda()
    N, n = g3["tab"].n_states, len(trajs)
    d_amp = torch.zeros(n * 2 * N, dtype=torch.float64, device="cuda")
    d_cls = torch.zeros(n * 6, dtype=torch.float64, device="cuda")
    d_diag = torch.zeros(n * 8, dtype=torch.float64, device="cuda")
    plan.run_device(d_init.data_ptr(), n, d_amp.data_ptr(), d_cls.data_ptr(), d_diag.data_ptr())
    plan.sync()
    assert plan.engine()[0] == mq.ENGINE_RESIDENT
    # the same cluster size and arithmetic: the device-buffer run repeats the host-buffer one
    assert np.array_equal(d_amp.cpu().numpy().reshape(n, 2 * N), amp1)
    assert np.array_equal(d_diag.cpu().numpy().reshape(n, 8), diag1)
    with pytest.raises(mq.MqctError):
        plan.set_cluster(9)
    plan.close()


def test_asym_top_system_matches_per_trajectory_kernel(mq, gpu_available, c2_tables):
    s, trajs, tab = c2_tables["s"], c2_tables["trajs"], c2_tables["tab"]
    a_rs, _, d_rs, eng, shape = _run(mq, tab, trajs, mq.PROP_FP32, mq.ENGINE_RESIDENT)
    assert eng == mq.ENGINE_RESIDENT and shape[0] >= 2
    a_pt, _, d_pt, _, _ = _run(mq, tab, trajs, mq.PROP_FP64, mq.ENGINE_PER_TRAJECTORY)
    p_rs = mq.channel_probabilities(a_rs, s.indx_chann, s.n_channels)
    p_pt = mq.channel_probabilities(a_pt, s.indx_chann, s.n_channels)
    assert np.max(np.abs(p_rs - p_pt)) < 2e-4
    assert np.all(d_rs[:, 4] == 0)
    assert np.allclose(d_rs[:, 1], d_pt[:, 1], rtol=1e-3)  # step counts
    a32, _, _, _, _ = _run(mq, tab, trajs, mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY)
    p32 = mq.channel_probabilities(a32, s.indx_chann, s.n_channels)
    assert np.max(np.abs(p_rs - p32)) < 5e-5
    a8, _, _, e8, sh8 = _run(mq, tab, trajs, mq.PROP_FP32, mq.ENGINE_RESIDENT, cluster=8)
    assert e8 == mq.ENGINE_RESIDENT and sh8[0] == 8
    p8 = mq.channel_probabilities(a8, s.indx_chann, s.n_channels)
    assert np.max(np.abs(p8 - p_rs)) < 5e-5


def test_start_beyond_the_grid(mq, oracle, gpu_available, g3):
    """Trajectories that start outside the R grid (the matrix is zero above R_max: no knot
    rows, y = 0) enter it and leave again: the resident engine against the oracle (FP64)
    and the FP32 per-trajectory kernel."""
    R = g3["tab"].R
    r0 = float(R[-1]) + 4.0
    base = g3["trajs"][::9][:12]
    trajs = [mq.Trajectory(t.e_coll, t.l_real, t.s_st, t.dt, r0, r0, time_lim=t.time_lim)
             for t in base]
    amp, cls, diag, eng, _ = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_RESIDENT)
    assert eng == mq.ENGINE_RESIDENT
    a2, c2, d2, _, _ = _run(mq, g3["tab"], trajs, mq.PROP_FP32, mq.ENGINE_PER_TRAJECTORY)
    oamp, ocls, odiag = _oracle_run(oracle, g3["otab"], trajs)
    idx = g3["s"].indx_chann
    p = mq.channel_probabilities(amp, idx, 10)
    assert np.max(np.abs(p - mq.channel_probabilities(oamp, idx, 10))) < 2e-4
    assert np.max(np.abs(p - mq.channel_probabilities(a2, idx, 10))) < 5e-5
    assert np.array_equal(diag[:, 4], odiag[:, 4])
    assert np.allclose(diag[:, 1], odiag[:, 1], rtol=1e-3)
