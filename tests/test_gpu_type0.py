"""GPU parity of the two-rotor (SYS_TYPE 0) matrix build: the basis is
orthonormal on the 5-D grid (constant surface), the FP64 form matches the oracle
on the 81-term SITES2 surface, and the split-precision forms stay within the
bounds of the rotor + atom builds."""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

GRID_KAT = (12, 4, 0, 12, 4, 4, 1)      # 9 216 points
GRID = (8, 4, 0, 8, 4, 4, 1)            # 4 096 points


def _system(mq, oracle=None):
    chans = [a + b for a in syn.asym_channels(1) for b in syn.asym_channels(1)]
    s = mq.CollisionSystem(0, chans, A=27.9, B=14.5, C=9.3)
    if oracle is None:
        return s, None
    ch = s.channels
    osys = oracle.OracleSystem(0, ch[:, 0], ch[:, 1], ch[:, 2], ch[:, 3], ch[:, 4], ch[:, 5],
                               e_ch=s.e_ch, vec1=s.vec1.reshape(-1), vec2=s.vec2.reshape(-1),
                               ldv=s.ldv)
    return s, osys


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("f16x3", 1e-5), ("bf16x3", 1e-3)])
def test_type0_constant_surface_gives_identity(mq, gpu_available, prec, tol):
    s, _ = _system(mq)
    R = np.array([5.0, 6.0, 7.0, 8.0])
    G = 12 * 4 * 12 * 4 * 4
    pes = dict(kind=0, n_terms=0, params=np.zeros(1), sites1=None, sites2=None,
               table=np.ones(len(R) * G))
    pr = {"fp64": mq.PREC_FP64, "f16x3": mq.PREC_F16X3, "bf16x3": mq.PREC_BF16X3}[prec]
    m, _, _ = mq.build_matrix(s, R, GRID_KAT, pes, precision=pr, mij_cutoff=0.0)
    m = m / syn.CM_TO_HARTREE
    diag = s.ind_mat[:, 0] == s.ind_mat[:, 1]
    assert np.max(np.abs(m[diag] - 1.0)) < tol
    assert np.max(np.abs(m[~diag])) < tol


def test_type0_fp64_matches_oracle_sites2(mq, oracle, gpu_available):
    s, osys = _system(mq, oracle)
    R = mq.r_grid(12, 5.0, 12.0)
    pd = syn.site_pes2()
    m, y2, sk = mq.build_matrix(s, R, GRID, pd, precision=mq.PREC_FP64, mij_cutoff=0.0)
    opes = oracle.OraclePes(pd["kind"], pd["n_terms"], pd["params"], sites1=pd["sites1"],
                            sites2=pd["sites2"])
    mref, y2ref, _ = oracle.build_matrix(osys, osys.states(), s.ind_mat, R, GRID, opes, mij_cut=0.0)
    rowmax = np.abs(mref).max(axis=1, keepdims=True)
    g = np.abs(mref).max()
    assert np.all(np.abs(m - mref) <= 1e-10 * rowmax + 1e-13 * g)
    assert np.max(np.abs(y2 - y2ref)) <= 1e-9 * np.abs(y2ref).max()


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
def test_type0_split_precision_matches_fp64(mq, gpu_available, prec):
    s, _ = _system(mq)
    R = mq.r_grid(12, 5.0, 12.0)
    pd = syn.site_pes2()
    m64, _, _ = mq.build_matrix(s, R, GRID, pd, precision=mq.PREC_FP64, mij_cutoff=0.0)
    pr = mq.PREC_F16X3 if prec == "f16x3" else mq.PREC_BF16X3
    m3, _, _ = mq.build_matrix(s, R, GRID, pd, precision=pr, mij_cutoff=0.0)
    rowmax = np.abs(m64).max(axis=1)
    g = rowmax.max()
    d = np.abs(m3 - m64)
    assert np.all(d <= 2e-3 * rowmax[:, None] + 2e-5 * g)
    sig = rowmax >= 1e-9 * g
    ek = d.max(axis=1)[sig] / rowmax[sig]
    if prec == "f16x3":
        assert np.median(ek) < 5e-6 and ek.max() < 5e-5, (np.median(ek), ek.max())
    else:
        assert np.median(ek) < 5e-5, np.median(ek)
