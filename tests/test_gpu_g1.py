"""The reference's two-run H2O + H2O AT-MQCT example (SYS_TYPE 0) through the
library alone: expansion-path matrices on the GPU (against the oracle), the
first run's SAVE_TRAJECT paths recorded by the GPU propagation (against the
reference's own AT_APPROX_TRAJS files), and the AT-MQCT second run along those
paths (against the reference's OPACITY_FUNCTIONS_L.out and cross sections).

Tolerances: matrices 1e-12 of the largest element (FP64, summation order);
records 1e-9 relative (FP64 RK4 of the same discretisation); FP64 probabilities
2e-7 relative (the golden file prints 8 digits) and cross sections 1e-8; FP32
arithmetic cross sections 1e-3 relative of the reference's."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def g1(mq, oracle, gpu_available):
    g = np.load(os.path.join(GOLD, "g1_h2o_h2o_at.npz"))
    A, B, Cc = float(g["A"]), float(g["B"]), float(g["C"])
    out = dict(g=g)
    for key, chans in (("s1", g["channels"][:1]), ("s9", g["channels"])):
        s = mq.CollisionSystem(0, chans, A=A, B=B, C=Cc)
        m, y2, sk = mq.build_matrix_expansion(s, g["R"], g["labels"], g["terms"], e_unit="KCAL",
                                              mij_cutoff=0.0)
        ch = s.channels
        osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                                   e_ch=s.e_ch, vec1=s.vec1.reshape(-1),
                                   vec2=s.vec2.reshape(-1), ldv=s.ldv)
        mo = oracle.expansion_matrix_type0(osys, osys.states(), s.ind_mat, g["labels"],
                                           g["terms"], mq.E_UNIT["KCAL"])
        out[key] = (s, m, mo)
    trajs1, meta = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), float(g["mass_red"]), 1,
                                     float(g["time_step1"]), float(g["rmax"]), dl=int(g["dl"]),
                                     time_lim=float(g["time_lim"]))
    s1, m1, _ = out["s1"]
    tab1 = mq.PropagationTables.from_system(s1, g["R"], m1, float(g["mass_red"]))
    _, _, diag1, paths = mq.propagate_record(tab1, trajs1, arith=mq.PROP_FP64)
    s9, m9, _ = out["s9"]
    tab9 = mq.PropagationTables.from_system(s9, g["R"], m9, float(g["mass_red"]))
    trajs2, _ = mq.trajectory_set(float(g["U"]), float(g["b_impct"]), float(g["mass_red"]), 1,
                                  float(g["time_step2"]), float(g["rmax"]), dl=int(g["dl"]),
                                  time_lim=float(g["time_lim"]))
    out.update(meta=meta, trajs1=trajs1, diag1=diag1, paths=paths, tab9=tab9, trajs2=trajs2)
    return out


def test_expansion_matrices_match_oracle(g1):
    for key, n_pairs in (("s1", 1), ("s9", 594)):
        s, m, mo = g1[key]
        assert s.P == n_pairs
        assert np.max(np.abs(m - mo)) <= 1e-12 * np.abs(mo).max()


def test_recorded_paths_equal_reference_files(g1):
    g = g1["g"]
    assert [t.l_real for t in g1["trajs1"]] == [float(l) for l in g["l"]]
    for i, rec in enumerate(g1["paths"]):
        assert len(rec) == g["n_rec"][i]
        h = len(rec) // 2
        for mine, ref in ((rec[:4], g["rec_head"][i]), (rec[h - 1:h + 2], g["rec_mid"][i]),
                          (rec[-3:], g["rec_tail"][i])):
            assert np.max(np.abs(mine - ref) / np.maximum(np.abs(ref), 1e-300)) <= 1e-9
        assert g1["diag1"][i, 1] == len(rec) - 1          # steps = records - 1


@pytest.mark.parametrize("arith", ["fp64", "fp32"])
def test_at_run_matches_reference(mq, g1, arith):
    g, meta = g1["g"], g1["meta"]
    ar = mq.PROP_FP64 if arith == "fp64" else mq.PROP_FP32
    amp, _, diag = mq.propagate(g1["tab9"], g1["trajs2"], arith=ar, mode=mq.MODE_AT,
                                at_paths=g1["paths"])
    s9 = g1["s9"][0]
    prob = mq.channel_probabilities(amp, s9.indx_chann, 9)
    sig = mq.cross_sections(prob, 0, meta["J_down"], meta["J_up"], meta["L_min"], meta["k"],
                            dl=meta["dl"])
    ref_p = g["opacity2"][:, 2:]
    if arith == "fp64":
        assert np.max(np.abs(prob - ref_p) / ref_p) < 2e-7
        assert np.allclose(sig, g["sigma2_mproj"], rtol=1e-8, atol=0)
    else:
        assert np.allclose(sig, g["sigma2_mproj"], rtol=1e-3, atol=0)


def test_cross_sections_on_the_device(mq, g1):
    """INELAST_CALC on the GPU from device amplitudes: channel probabilities, the
    J-resolved cross sections of PARTIAL_CROSS_SECTIONS_J.out and their sums."""
    import torch
    g, meta = g1["g"], g1["meta"]
    amp, _, _ = mq.propagate(g1["tab9"], g1["trajs2"], arith=mq.PROP_FP64, mode=mq.MODE_AT,
                             at_paths=g1["paths"])
    s9 = g1["s9"][0]
    d_amp = torch.from_numpy(amp).cuda()
    prob, partial, sigma = mq.cross_sections_device(d_amp, s9, 0, meta["J_down"], meta["J_up"],
                                                    meta["L_min"], meta["k"], dl=meta["dl"])
    torch.cuda.synchronize()
    p_host = mq.channel_probabilities(amp, s9.indx_chann, 9)
    assert np.allclose(prob.cpu().numpy(), p_host, rtol=1e-14, atol=1e-16)
    s_host = mq.cross_sections(p_host, 0, meta["J_down"], meta["J_up"], meta["L_min"], meta["k"],
                               dl=meta["dl"])
    assert np.allclose(sigma.cpu().numpy(), s_host, rtol=1e-13)
    ref = g["partial2"][:, 1:]
    assert partial.shape == ref.shape
    assert np.max(np.abs(partial.cpu().numpy() - ref) / ref) < 2e-7
    assert np.allclose(sigma.cpu().numpy(), g["sigma2_mproj"], rtol=1e-8)


def test_at_adaptive_step_matches_oracle(mq, oracle, g1):
    """AT_ADAPT_STP on the GPU (RK4 steps from the coupling energy along each saved
    path, AT_ADAPTOL = 5e-4, TIME_STEP the smallest step) against the oracle's
    restatement on the same paths: the same number of steps and the same end time,
    probabilities within 1e-8 (FP64)."""
    g = g1["g"]
    tab = g1["tab9"]
    trajs = g1["trajs2"][:6]
    paths = g1["paths"][:6]
    amp, _, diag = mq.propagate(tab, trajs, arith=mq.PROP_FP64, mode=mq.MODE_AT,
                                at_paths=paths,
                                integrator=("AT_ADAPT", 5e-4, float(g["time_step2"])))
    otab = oracle.OracleTables(tab.j12, tab.m12, tab.ej, tab.ind_mat, tab.R, tab.mat, tab.y2,
                               tab.mass_au)
    N = len(tab.j12)
    for i, t in enumerate(trajs):
        tr = oracle.make_traj(t.e_coll, t.l_real, t.s_st, t.dt, t.r_start, t.r_fin,
                              time_lim=t.time_lim, method=2, eps=5e-4,
                              hmin=float(g["time_step2"]))
        oamp, odiag = oracle.dotraject_at(otab, tr, paths[i])
        assert diag[i, 1] == odiag[1]
        assert diag[i, 0] == pytest.approx(odiag[0], rel=1e-12)
        p = amp[i, :N] ** 2 + amp[i, N:] ** 2
        po = oamp[:N] ** 2 + oamp[N:] ** 2
        assert np.max(np.abs(p - po)) < 1e-8
