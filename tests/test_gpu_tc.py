"""GPU parity of the split-precision tcgen05 contractions (BF16x3, F16x3)
against the FP64 forms.

Split precision is judged two ways:
 - element level: for every element |dM_k(R)| <= 2e-3 * max_R |M_k| + 2e-5 *
   max |M| (both modes), and over pairs that do not vanish by symmetry the
   relative max-norm error e_k = max_R |dM_k| / max_R |M_k|: BF16x3 median
   <= 5e-5 (per entry), F16x3 median <= 5e-6 and max <= 5e-5;
 - physics level: inelastic cross sections from the
   split-precision matrix within 1e-3 relative of those from the FP64 matrix.
"""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _errors(m3, m64):
    rowmax = np.abs(m64).max(axis=1, keepdims=True)
    g = np.abs(m64).max()
    d = np.abs(m3 - m64)
    assert np.all(d <= 2e-3 * rowmax + 2e-5 * g), np.max(d / (2e-3 * rowmax + 2e-5 * g))
    sig = rowmax[:, 0] >= 1e-9 * g
    big = (np.abs(m64) >= 1e-3 * rowmax) & sig[:, None]
    rel = d[big] / np.abs(m64[big])
    ek = d.max(axis=1)[sig] / rowmax[sig, 0]
    return float(np.median(rel)), float(np.quantile(rel, 0.99)), float(np.median(ek)), float(ek.max())


def _c2_small(mq, jmax=3):
    chans = [c for c in syn.config_c2()["channels"] if c[0] <= jmax]
    return mq.CollisionSystem(4, chans, A=27.9, B=14.5, C=9.3)


@pytest.mark.parametrize("grid,nR", [((16, 16, 0, 0, 0, 0, 1), 37), ((12, 12, 6, 0, 0, 0, 1), 37),
                                     ((16, 16, 4, 0, 0, 0, 1), 300), ((8, 24, 0, 0, 0, 0, 1), 200)])
@pytest.mark.parametrize("prec", ["bf16x3", "f16x3"])
def test_split_precision_matches_fp64_type4(mq, gpu_available, grid, nR, prec):
    s = _c2_small(mq)
    R = mq.r_grid(nR, 3.0, 25.0)
    pes = syn.site_pes(12, seed=2)
    m64, _, _ = mq.build_matrix(s, R, grid, pes, precision=mq.PREC_FP64, mij_cutoff=0.0)
    pr = mq.PREC_BF16X3 if prec == "bf16x3" else mq.PREC_F16X3
    m3, _, _ = mq.build_matrix(s, R, grid, pes, precision=pr, mij_cutoff=0.0)
    med, p99, ek_med, ek_max = _errors(m3, m64)
    if prec == "bf16x3":
        assert med < 5e-5, med
    else:
        assert ek_med < 5e-6 and ek_max < 5e-5, (ek_med, ek_max)


@pytest.mark.parametrize("prec", ["bf16x3", "f16x3"])
def test_split_precision_matches_oracle_type1(mq, oracle, gpu_available, prec):
    c1 = syn.config_c1()
    s = mq.CollisionSystem(1, c1["channels"], BE=c1["BE"])
    R = mq.r_grid(c1["nR"], c1["rmin"], c1["rmax"])
    pr = mq.PREC_BF16X3 if prec == "bf16x3" else mq.PREC_F16X3
    m3, y3, _ = mq.build_matrix(s, R, c1["grid"], c1["pes"], precision=pr, mij_cutoff=0.0)
    osys = oracle.OracleSystem(1, s.channels[:, 0], e_ch=s.e_ch, vec1=np.ones(s.n_channels), ldv=1)
    pes = oracle.OraclePes(c1["pes"]["kind"], c1["pes"]["n_terms"], c1["pes"]["params"])
    mref, _, _ = oracle.build_matrix(osys, osys.states(), s.ind_mat, R, c1["grid"], pes, mij_cut=0.0)
    med, _, ek_med, ek_max = _errors(m3, mref)
    if prec == "bf16x3":
        assert med < 5e-5
    else:
        assert ek_med < 5e-6 and ek_max < 5e-5, (ek_med, ek_max)


@pytest.mark.parametrize("prec", ["bf16x3", "f16x3"])
def test_split_precision_cross_sections_within_1e3(mq, gpu_available, prec):
    """Asymmetric top + atom (j <= 3, 84 states), 36 trajectories at 500 cm^-1:
    inelastic cross sections from the split-precision matrix vs from the FP64 matrix
    (both propagated in FP64).  The site-site wall keeps every turning point
    inside the R grid."""
    s = _c2_small(mq)
    R = mq.r_grid(120, 3.0, 25.0)
    pes = syn.site_pes(12, seed=2)
    sig = {}
    split = mq.PREC_BF16X3 if prec == "bf16x3" else mq.PREC_F16X3
    for pr in (mq.PREC_FP64, split):
        mat, _, _ = mq.build_matrix(s, R, (24, 24, 0, 0, 0, 0, 1), pes, precision=pr)
        tab = mq.PropagationTables.from_system(s, R, mat, 3.7523705333)
        trajs, meta = mq.trajectory_set(500.0, 12.0, 3.7523705333, 1, 10.0, 25.0)
        trajs = trajs[::max(1, len(trajs) // 36)]
        amp, cls, diag = mq.propagate(tab, trajs, arith=mq.PROP_FP64)
        assert np.all(diag[:, 4] == 0)
        p = mq.channel_probabilities(amp, s.indx_chann, s.n_channels)
        l = np.array([t.l_real for t in trajs])
        sig[pr] = ((2 * l + 1)[:, None] * p).sum(axis=0)
    a, b = sig[split], sig[mq.PREC_FP64]
    big = b > 1e-4 * b[1:].max()
    big[0] = False  # elastic channel
    assert big.sum() >= 3
    assert np.max(np.abs(a[big] - b[big]) / b[big]) < 1e-3


def test_tc_plan_reports_flops_and_timing(mq, gpu_available):
    import torch
    s = _c2_small(mq)
    R = mq.r_grid(64, 3.0, 25.0)
    plan = mq.MatrixPlan(s, R, (16, 16, 2, 0, 0, 0, 1), syn.site_pes(12, seed=2),
                         precision=mq.PREC_BF16X3)
    assert plan.flops == pytest.approx(3 * 2.0 * s.P * len(R) * 16 * 16 * 2)
    d = torch.empty(s.P * len(R), dtype=torch.float64, device="cuda")
    plan.execute(d.data_ptr())
    plan.sync()
    t = plan.timing()
    assert all(x > 0 for x in t)
    plan.close()


@pytest.mark.parametrize("grid", [(12, 12, 8, 0, 0, 0, 1), (16, 16, 0, 0, 0, 0, 1)])
def test_epilogue_layouts_agree_and_tune(mq, gpu_available, grid):
    """The 8- and 16-warp epilogue layouts of the contraction give bitwise identical
    matrices (every column's sum has the same order); mqct_matrix_plan_tune times both,
    keeps one of them and its build equals them."""
    import torch
    s = _c2_small(mq)
    R = mq.r_grid(300, 3.0, 25.0)
    plan = mq.MatrixPlan(s, R, grid, syn.site_pes(12, seed=2), precision=mq.PREC_F16X3)
    n = s.P * len(R)
    out = {}
    for w in (8, 16, 0):
        plan.set_epilogue(w)
        m = torch.empty(n, dtype=torch.float64, device="cuda")
        y = torch.empty_like(m)
        sk = torch.empty(s.P, dtype=torch.int32, device="cuda")
        plan.execute(m.data_ptr(), y.data_ptr(), sk.data_ptr())
        plan.sync()
        out[w] = (m.cpu(), y.cpu(), sk.cpu())
    # the default rule: 16 warps with several accumulation groups per chunk, else 8
    assert plan.epilogue()[0] == (16 if grid[2] > 2 else 8)
    m = torch.empty(n, dtype=torch.float64, device="cuda")
    plan.tune(m.data_ptr())
    plan.sync()
    w, ms = plan.epilogue()
    assert w in (8, 16) and ms[0] > 0 and ms[1] > 0
    for k in range(3):
        assert torch.equal(out[8][k], out[16][k]) and torch.equal(out[0][k], out[8][k])
    assert torch.equal(m.cpu(), out[8][0])
    with pytest.raises(mq.MqctError):
        plan.set_epilogue(12)
    plan.close()
