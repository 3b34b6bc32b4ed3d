"""GPU parity of the matrix build (C ABI mqct_build_matrix) against the FP64
oracle on seeded inputs.

Tolerances: the FP64 form must agree to |dM| <= 1e-11 * max_R |M_k| (summation
order only); the BF16x3 tensor-core form to the split-precision bound stated
in the test (relative error against max(|M|, 1e-3 max_R |M_k|))."""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _oracle_system(oracle, s):
    ch = s.channels
    if s.sys_type == 1:
        return oracle.OracleSystem(1, ch[:, 0], e_ch=s.e_ch, vec1=np.ones(len(ch)), ldv=1)
    return oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch,
                               vec1=s.vec1.reshape(-1), ldv=s.ldv)


def _oracle_build(oracle, s, R, grid, pes_d, cut=1e-12):
    osys = _oracle_system(oracle, s)
    states = osys.states()
    pes = oracle.OraclePes(pes_d["kind"], pes_d["n_terms"], pes_d["params"], sites1=pes_d.get("sites1"))
    return oracle.build_matrix(osys, states, s.ind_mat, R, grid, pes, mij_cut=cut)


def _c2_small(mq, jmax=3):
    chans = [c for c in syn.config_c2()["channels"] if c[0] <= jmax]
    return mq.CollisionSystem(4, chans, A=27.9, B=14.5, C=9.3)


def _assert_close(m_gpu, m_ref, rel, floor=1e-14):
    """|dM_k| <= rel * max_R |M_k| + floor * max |M|: elements that vanish by
    symmetry carry only the rounding noise of the global scale."""
    bound = rel * np.abs(m_ref).max(axis=1, keepdims=True) + floor * np.abs(m_ref).max()
    excess = np.abs(m_gpu - m_ref) / bound
    assert np.max(excess) <= 1.0, np.max(excess)


def _check_spline(oracle, R, mat, y2):
    """The GPU spline of the GPU values equals the oracle spline of those values."""
    for k in range(0, mat.shape[0], max(1, mat.shape[0] // 50)):
        c = mat[k]
        ref = oracle.spline(R, c, (c[1] - c[0]) / (R[1] - R[0]), (c[-1] - c[-2]) / (R[-1] - R[-2]))
        assert np.allclose(y2[k], ref, rtol=1e-10, atol=1e-12 * (np.abs(ref).max() + 1e-300))


def _assert_skips(sk, skref, mref_raw_cm, R, cut_cm, noise_cm):
    """MIJ_CUTOFF flags must agree wherever the decision is not within the
    rounding noise of the cutoff."""
    ir1, ir2 = np.argmin(np.abs(R - 6.0)), np.argmin(np.abs(R - 8.0))
    v = np.maximum(np.abs(mref_raw_cm[:, ir1]), np.abs(mref_raw_cm[:, ir2]))
    robust = np.abs(v - cut_cm) > 10 * noise_cm
    assert np.array_equal(sk[robust], skref[robust])


def test_c1_fp64_matches_oracle(mq, oracle, gpu_available):
    c1 = syn.config_c1()
    s = mq.CollisionSystem(1, c1["channels"], BE=c1["BE"])
    R = mq.r_grid(c1["nR"], c1["rmin"], c1["rmax"])
    mat, y2, sk = mq.build_matrix(s, R, c1["grid"], c1["pes"], precision=mq.PREC_FP64)
    mref, y2ref, skref = _oracle_build(oracle, s, R, c1["grid"], c1["pes"])
    assert (s.P, len(R)) == (506, 200)
    noise = 1e-13 * np.abs(mref).max() / syn.CM_TO_HARTREE
    raw, _, _ = _oracle_build(oracle, s, R, c1["grid"], c1["pes"], cut=0.0)
    _assert_skips(sk, skref, raw / syn.CM_TO_HARTREE, R, 1e-12, noise)
    both = (sk == 0) & (skref == 0)
    _assert_close(mat[both], mref[both], 1e-11)
    _assert_close(y2[both], y2ref[both], 1e-9, floor=1e-10)
    _check_spline(oracle, R, mat[both], y2[both])


@pytest.mark.parametrize("grid", [(16, 16, 0, 0, 0, 0, 1), (12, 12, 6, 0, 0, 0, 1),
                                  (10, 14, 0, 0, 0, 0, 0)])
def test_c2_small_fp64_matches_oracle(mq, oracle, gpu_available, grid):
    s = _c2_small(mq)
    R = mq.r_grid(37, 3.0, 25.0)
    pes = syn.site_pes(12, seed=2)
    mat, y2, sk = mq.build_matrix(s, R, grid, pes, precision=mq.PREC_FP64, mij_cutoff=0.0)
    mref, y2ref, skref = _oracle_build(oracle, s, R, grid, pes, cut=0.0)
    _assert_close(mat, mref, 1e-11)
    # y2 of symmetry-zero rows is the spline of rounding noise (amplified by 1/h^2)
    _assert_close(y2, y2ref, 1e-9, floor=1e-10)
    _check_spline(oracle, R, mat, y2)
    # with the reference's default cutoff (1e-12 cm^-1)
    mat_c, _, sk = mq.build_matrix(s, R, grid, pes, precision=mq.PREC_FP64)
    _, _, skref = _oracle_build(oracle, s, R, grid, pes)
    _assert_skips(sk, skref, mref / syn.CM_TO_HARTREE, R, 1e-12,
                  1e-13 * np.abs(mref).max() / syn.CM_TO_HARTREE)
    assert np.all(mat_c[sk == 1] == 0)


def test_mij_cutoff_zeroes_and_flags(mq, oracle, gpu_available):
    s = _c2_small(mq, jmax=2)
    R = mq.r_grid(21, 3.0, 25.0)
    pes = syn.site_pes(12, seed=2)
    cut = 5.0  # cm^-1: large enough to drop several elements
    mat, y2, sk = mq.build_matrix(s, R, (8, 8, 0, 0, 0, 0, 1), pes, precision=mq.PREC_FP64,
                                  mij_cutoff=cut)
    mref, _, skref = _oracle_build(oracle, s, R, (8, 8, 0, 0, 0, 0, 1), pes, cut=cut)
    raw, _, _ = _oracle_build(oracle, s, R, (8, 8, 0, 0, 0, 0, 1), pes, cut=0.0)
    assert sk.sum() > 0
    _assert_skips(sk, skref, raw / syn.CM_TO_HARTREE, R, cut,
                  1e-13 * np.abs(raw).max() / syn.CM_TO_HARTREE)
    assert np.all(mat[sk == 1] == 0) and np.all(y2[sk == 1] == 0)


def test_plan_reuse_is_deterministic(mq, gpu_available):
    import torch
    s = _c2_small(mq)
    R = mq.r_grid(33, 3.0, 25.0)
    plan = mq.MatrixPlan(s, R, (12, 12, 0, 0, 0, 0, 1), syn.site_pes(12, seed=2),
                         precision=mq.PREC_FP64)
    out = [torch.zeros(s.P * len(R), dtype=torch.float64, device="cuda") for _ in range(2)]
    for o in out:
        plan.execute(o.data_ptr())
    plan.sync()
    assert torch.equal(out[0], out[1])
    plan.close()


def test_pinned_output_arrays_match_pageable(mq, gpu_available):
    """mqct_build_matrix into pinned host arrays (the copy engine writes them directly) gives
    the results it writes into pageable arrays (staged through the library's pinned slots);
    the c2 system at j <= 6 is large enough for the staged path (Mat_el above 16 MB)."""
    import torch
    s = _c2_small(mq, jmax=6)
    R = mq.r_grid(300, 3.0, 25.0)
    assert s.P * len(R) * 8 > 16 << 20
    args = (s, R, (12, 12, 0, 0, 0, 0, 1), syn.site_pes(12, seed=2))
    ref = mq.build_matrix(*args, precision=mq.PREC_FP64)
    pinned = (torch.empty((s.P, len(R)), dtype=torch.float64, pin_memory=True),
              torch.empty((s.P, len(R)), dtype=torch.float64, pin_memory=True),
              torch.empty(s.P, dtype=torch.int32, pin_memory=True))
    got = mq.build_matrix(*args, precision=mq.PREC_FP64, out=tuple(t.numpy() for t in pinned))
    mq.release_cached_build()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
