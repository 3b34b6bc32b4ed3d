"""Split-precision accuracy on the headline build as written: the asymmetric top + atom
system with the full j <= 8 basis (969 states, 31 977 pairs) on the 48 GL beta x 48 gamma
x 48 alpha grid (K = 110 592 points per element), at a handful of R points spread over
3-25 bohr (the repulsive wall included).

Error metrics, against the FP64 form of the same build (mma.sync f64):
 - e_k = max_R |dM_k| / max_R |M_k| per element (the relative error of the radial
   function), over the pairs that do not vanish by symmetry;
 - per entry |dM| / |M| for the entries above 1e-3 of their element's maximum.
The F16x3 contraction drains its FP32 tensor-core accumulators into FP64 sums after
every 64-point chunk of every alpha point, so the long FP32 accumulations that lost
bits on the as-written grid are gone; what remains is the 22-bit split of the
operands.  A seeded sample of elements is also checked against the oracle's literal
restatement of INTEGRATOR_TEMP, and cross sections from an F16x3 matrix (FP64
propagation) against those from the FP64 matrix."""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

R_POINTS = [3.0, 3.5, 4.5, 6.0, 8.0, 12.0, 18.0, 25.0]


def _system(mq):
    c2 = syn.config_c2(alpha_grid=True)
    s = mq.CollisionSystem(4, c2["channels"], A=c2["A"], B=c2["B"], C=c2["C"])
    return c2, s


def _metrics(m1, m0):
    rowmax = np.abs(m0).max(axis=1)
    sig = rowmax >= 1e-9 * rowmax.max()
    d = np.abs(m1 - m0)
    ek = d.max(axis=1)[sig] / rowmax[sig]
    big = (np.abs(m0) >= 1e-3 * rowmax[:, None]) & sig[:, None]
    rel = d[big] / np.abs(m0[big])
    return ek, rel


def test_c2_as_written_f16x3_against_fp64(mq, gpu_available):
    c2, s = _system(mq)
    R = np.array(R_POINTS)
    m64, _, _ = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=mq.PREC_FP64,
                                mij_cutoff=0.0)
    m16, _, _ = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=mq.PREC_F16X3,
                                mij_cutoff=0.0)
    ek, rel = _metrics(m16, m64)
    assert np.max(ek) <= 1e-4, (np.median(ek), np.quantile(ek, 0.99), np.max(ek))
    assert np.quantile(rel, 0.99) <= 1e-4, (np.median(rel), np.quantile(rel, 0.99))
    mq.release_cached_build()


def test_c2_as_written_fp64_form_against_oracle(mq, oracle, gpu_available):
    """A seeded sample of elements at three R points: the FP64 GPU form against the
    oracle's literal INTEGRATOR_TEMP (wavefunctions re-evaluated at every point of the
    110 592-point grid), and the F16x3 form within 1e-4 of each element's maximum."""
    c2, s = _system(mq)
    R = np.array([3.5, 6.0, 12.0])
    m64, _, _ = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=mq.PREC_FP64,
                                mij_cutoff=0.0)
    m16, _, _ = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=mq.PREC_F16X3,
                                mij_cutoff=0.0)
    ch = s.channels
    osys = oracle.OracleSystem(4, ch[:, 0], ch[:, 1], ch[:, 2], e_ch=s.e_ch,
                               vec1=s.vec1.reshape(-1), ldv=s.ldv)
    pd = c2["pes"]
    pes = oracle.OraclePes(pd["kind"], pd["n_terms"], pd["params"], sites1=pd["sites1"])
    rng = np.random.default_rng(11)
    sel = np.sort(rng.choice(s.P, 24, replace=False))
    ref = oracle.integrate_elements(osys, osys.states(), np.ascontiguousarray(s.ind_mat[sel]), R,
                                    c2["grid"], pes, literal=True) * syn.CM_TO_HARTREE
    scale = np.abs(m64).max()
    assert np.max(np.abs(m64[sel] - ref)) <= 1e-11 * scale
    rowmax = np.abs(ref).max(axis=1, keepdims=True)
    # elements that vanish by symmetry carry rounding noise only: absolute floor 1e-8 of
    # the largest element (the floor of the per-entry error metric)
    assert np.all(np.abs(m16[sel] - ref) <= 1e-4 * rowmax + 1e-8 * scale)
    mq.release_cached_build()


def test_c2_as_written_cross_sections_within_1e3(mq, gpu_available):
    """Cross sections from the as-written F16x3 matrix (100 R points, FP64 propagation
    of 48 trajectories at 500 cm^-1 from the ground state) against those from the FP64
    matrix: within 1e-3 relative for every inelastic channel above 1e-4 of the largest."""
    c2, s = _system(mq)
    R = mq.r_grid(100, 3.0, 25.0)
    sig = {}
    for pr in (mq.PREC_FP64, mq.PREC_F16X3):
        mat, _, _ = mq.build_matrix(s, R, c2["grid"], c2["pes"], precision=pr)
        tab = mq.PropagationTables.from_system(s, R, mat, c2["mass_amu"])
        trajs, meta = mq.trajectory_set(500.0, 12.0, c2["mass_amu"], 1, 10.0, 25.0)
        trajs = trajs[::max(1, len(trajs) // 48)]
        amp, cls, diag = mq.propagate(tab, trajs, arith=mq.PROP_FP64)
        assert np.all(diag[:, 4] == 0)
        p = mq.channel_probabilities(amp, s.indx_chann, s.n_channels)
        l = np.array([t.l_real for t in trajs])
        sig[pr] = ((2 * l + 1)[:, None] * p).sum(axis=0)
    a, b = sig[mq.PREC_F16X3], sig[mq.PREC_FP64]
    big = b > 1e-4 * b[1:].max()
    big[0] = False
    assert big.sum() >= 5
    assert np.max(np.abs(a[big] - b[big]) / b[big]) < 1e-3
    mq.release_cached_build()
