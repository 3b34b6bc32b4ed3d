"""ctypes binding of the CPU FP64 oracle (oracle/mqct_oracle.c).

TEST INFRASTRUCTURE ONLY: loaded by tests/, the smoke check and the CPU
baseline leg of bench.py as the checker.  The product (mqct_b200) never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmqct_oracle.so")
_lib = None

i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class System(C.Structure):
    _fields_ = [("sys_type", C.c_int32), ("n_channels", C.c_int32),
                ("j1", C.c_void_p), ("ka1", C.c_void_p), ("kc1", C.c_void_p),
                ("j2", C.c_void_p), ("ka2", C.c_void_p), ("kc2", C.c_void_p),
                ("e_ch", C.c_void_p), ("vec1", C.c_void_p), ("vec2", C.c_void_p),
                ("ldv", C.c_int32)]


class Pes(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_terms", C.c_int32), ("p", C.c_void_p),
                ("n_sites1", C.c_int32), ("n_sites2", C.c_int32),
                ("sites1", C.c_void_p), ("sites2", C.c_void_p), ("table", C.c_void_p)]


class Grid(C.Structure):
    _fields_ = [("n_beta", C.c_int32), ("n_gamma", C.c_int32), ("n_alpha", C.c_int32),
                ("n_beta2", C.c_int32), ("n_alpha2", C.c_int32), ("n_gamma2", C.c_int32),
                ("eq_gamma", C.c_int32)]


class Tables(C.Structure):
    _fields_ = [("n_states", C.c_int32), ("j12", C.c_void_p), ("m12", C.c_void_p),
                ("ej", C.c_void_p), ("P", C.c_int64), ("ind_mat", C.c_void_p),
                ("nR", C.c_int32), ("R", C.c_void_p), ("mat", C.c_void_p),
                ("y2", C.c_void_p), ("mass_au", C.c_double)]


class Traj(C.Structure):
    _fields_ = [("e_coll", C.c_double), ("l_real", C.c_double), ("s_st", C.c_int32),
                ("dt", C.c_double), ("r_start", C.c_double), ("r_fin", C.c_double),
                ("numb_orb_prds", C.c_int32), ("numb_oscl_prds", C.c_int32),
                ("time_lim", C.c_double), ("max_steps", C.c_int64), ("method", C.c_int32),
                ("eps", C.c_double), ("hmin", C.c_double), ("cs", C.c_int32)]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_plgndr.restype = C.c_double
        L.orc_plgndr.argtypes = [C.c_int, C.c_int, C.c_double]
        L.orc_gauleg.argtypes = [C.c_int, f64p, f64p]
        L.orc_w3js.restype = C.c_double
        L.orc_w3js.argtypes = [C.c_int] * 6
        L.orc_cg.restype = C.c_double
        L.orc_cg.argtypes = [C.c_int] * 6
        L.orc_expansion_matrix_type8.argtypes = [C.POINTER(System), C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_djkm.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                               C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_wf_diat.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_wf_asym.argtypes = [C.c_int, f64p, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_asym_top.restype = C.c_int
        L.orc_asym_top.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.c_int, C.POINTER(C.c_double), f64p]
        L.orc_spline.argtypes = [f64p, f64p, C.c_int, C.c_double, C.c_double, f64p]
        L.orc_count_states.argtypes = [C.POINTER(System)]
        L.orc_enumerate_states.argtypes = [C.POINTER(System), i32p, i32p, i32p, f64p]
        L.orc_count_pairs.restype = C.c_int64
        L.orc_count_pairs.argtypes = [C.c_int, i32p]
        L.orc_ind_mat.restype = C.c_int64
        L.orc_ind_mat.argtypes = [C.c_int, i32p, i32p]
        L.orc_rgrid.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, f64p]
        L.orc_pes_eval.restype = C.c_double
        L.orc_pes_eval.argtypes = [C.POINTER(Pes)] + [C.c_double] * 7
        L.orc_build_matrix.argtypes = [C.POINTER(System), C.c_int, i32p, i32p, i32p, C.c_int64,
                                       i32p, C.c_int, f64p, C.POINTER(Grid), C.POINTER(Pes),
                                       C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_int64, C.c_int64, C.c_int, f64p, f64p, i32p]
        L.orc_integrate_elements.argtypes = [C.POINTER(System), C.c_int, i32p, i32p, i32p,
                                             C.c_int64, i32p, C.c_int, f64p, C.POINTER(Grid),
                                             C.POINTER(Pes), C.c_int, C.c_int64, C.c_int64,
                                             C.c_int, C.c_int, C.c_int, f64p]
        L.orc_write_mtrx_uf.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, i32p, C.c_int,
                                        C.c_int64, i32p, C.c_int, f64p, f64p]
        L.orc_read_mtrx_dat_header.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                               C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                               C.POINTER(C.c_int)]
        L.orc_read_mtrx_dat.argtypes = [C.c_char_p, C.c_int, i32p, i32p, f64p, f64p]
        L.orc_derivs.argtypes = [C.POINTER(Tables), C.c_double, f64p, f64p]
        L.orc_dotraject.argtypes = [C.POINTER(Tables), C.POINTER(Traj), f64p, f64p, f64p]
        L.orc_propagate_batch.argtypes = [C.POINTER(Tables), C.c_int, C.POINTER(Traj), C.c_int,
                                          f64p, f64p, f64p]
        L.orc_dotraject_at.argtypes = [C.POINTER(Tables), C.POINTER(Traj), C.c_int, f64p, f64p,
                                       f64p]
        L.orc_inelast.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, f64p,
                                  C.c_double, f64p]
        L.orc_inelast_dl.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_int, f64p, C.c_double, f64p]
        L.orc_dotraject_rec.argtypes = [C.POINTER(Tables), C.POINTER(Traj), f64p, f64p, f64p,
                                        f64p, C.c_int64, C.POINTER(C.c_int64)]
        L.orc_expansion_matrix_type0_identical.argtypes = [C.POINTER(System), C.c_void_p,
                                                          C.c_void_p, C.c_void_p, C.c_void_p,
                                                          C.c_int64, C.c_void_p, C.c_int,
                                                          C.c_void_p, C.c_int, C.c_void_p,
                                                          C.c_double, C.c_void_p]
        L.orc_expansion_matrix_atom.argtypes = [C.POINTER(System)] + [C.c_void_p] * 3 + [C.c_int64, C.c_void_p, C.c_int,
                                                C.c_void_p, C.c_int, C.c_void_p, C.c_double,
                                                C.c_void_p]
        L.orc_project_terms_atom.argtypes = [C.c_int, C.c_int, C.c_void_p] + [C.c_int] * 4 + [
            C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_expansion_term.argtypes = [C.c_int] * 6 + [C.c_double] * 5 + [
            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_project_terms.argtypes = [C.c_int, C.c_int, C.c_void_p] + [C.c_int] * 7 + [
            C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_expansion_matrix_type7.argtypes = [C.POINTER(System), C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_int, C.c_void_p, C.c_double,
                                                 C.c_void_p]
        L.orc_expansion_matrix_type0.argtypes = [C.POINTER(System), C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_int,
                                                 C.c_void_p, C.c_int, C.c_void_p, C.c_double,
                                                 C.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- helpers
def plgndr(l, m, x):
    return lib().orc_plgndr(l, m, x)


def gauleg(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauleg(n, x, w)
    return x, w


def djkm(j, k, m, a, b, g):
    re, im = C.c_double(), C.c_double()
    lib().orc_djkm(j, k, m, a, b, g, C.byref(re), C.byref(im))
    return re.value, im.value


def wf_diat(j, m, th, ph=0.0):
    re, im = C.c_double(), C.c_double()
    lib().orc_wf_diat(j, m, th, ph, C.byref(re), C.byref(im))
    return re.value, im.value


def wf_asym(j, coeff, m, a, b, g):
    re, im = C.c_double(), C.c_double()
    lib().orc_wf_asym(j, np.ascontiguousarray(coeff, dtype=np.float64), m, a, b, g,
                      C.byref(re), C.byref(im))
    return re.value, im.value


def asym_top(A, B, Cc, j, ka, kc):
    e = C.c_double()
    v = np.zeros(2 * j + 1)
    rc = lib().orc_asym_top(A, B, Cc, j, ka, kc, C.byref(e), v)
    if rc:
        raise ValueError(f"invalid asymmetric-top level j={j} ka={ka} kc={kc} ({rc})")
    return e.value, v


def cg(j1, j2, j3, m1, m2, m3):
    return lib().orc_cg(j1, j2, j3, m1, m2, m3)


def spline(x, y, yp1, ypn):
    y2 = np.zeros_like(x)
    lib().orc_spline(np.ascontiguousarray(x), np.ascontiguousarray(y), len(x), yp1, ypn, y2)
    return y2


def rgrid(n, rmin, rmax, equidistant=True):
    R = np.zeros(n)
    lib().orc_rgrid(n, rmin, rmax, 1 if equidistant else 0, R)
    return R


class OracleSystem:
    """Holds the numpy arrays behind an orc_system so that pointers stay valid."""

    def __init__(self, sys_type, j1, ka1=None, kc1=None, j2=None, ka2=None, kc2=None,
                 e_ch=None, vec1=None, vec2=None, ldv=1):
        def a32(x):
            return None if x is None else np.ascontiguousarray(x, dtype=np.int32)

        def a64(x):
            return None if x is None else np.ascontiguousarray(x, dtype=np.float64)

        self.arr = dict(j1=a32(j1), ka1=a32(ka1), kc1=a32(kc1), j2=a32(j2), ka2=a32(ka2),
                        kc2=a32(kc2), e_ch=a64(e_ch), vec1=a64(vec1), vec2=a64(vec2))
        self.s = System(sys_type, len(j1), *[_ptr(self.arr[k]) for k in
                                             ("j1", "ka1", "kc1", "j2", "ka2", "kc2", "e_ch",
                                              "vec1", "vec2")], ldv)

    def states(self):
        L = lib()
        n = L.orc_count_states(C.byref(self.s))
        ic = np.zeros(n, np.int32)
        j12 = np.zeros(n, np.int32)
        m12 = np.zeros(n, np.int32)
        ej = np.zeros(n)
        L.orc_enumerate_states(C.byref(self.s), ic, j12, m12, ej)
        return ic, j12, m12, ej


def ind_mat(m12):
    m12 = np.ascontiguousarray(m12, dtype=np.int32)
    L = lib()
    P = L.orc_count_pairs(len(m12), m12)
    ind = np.zeros(2 * P, np.int32)
    L.orc_ind_mat(len(m12), m12, ind)
    return ind.reshape(P, 2)


class OraclePes:
    def __init__(self, kind, n_terms, params, sites1=None, sites2=None, table=None):
        self.p = np.ascontiguousarray(params, dtype=np.float64)
        self.s1 = None if sites1 is None else np.ascontiguousarray(sites1, dtype=np.float64)
        self.s2 = None if sites2 is None else np.ascontiguousarray(sites2, dtype=np.float64)
        self.tab = None if table is None else np.ascontiguousarray(table, dtype=np.float64)
        self.s = Pes(kind, n_terms, _ptr(self.p),
                     0 if self.s1 is None else len(self.s1) // 3,
                     0 if self.s2 is None else len(self.s2) // 3,
                     _ptr(self.s1), _ptr(self.s2), _ptr(self.tab))

    def __call__(self, R, alpha=0.0, beta=0.0, gamma=0.0, aa=0.0, bb=0.0, gg=0.0):
        return lib().orc_pes_eval(C.byref(self.s), R, alpha, beta, gamma, aa, bb, gg)


def build_matrix(osys, states, ind, R, grid, pes, mij_cut=1e-12, r_cut1=6.0, r_cut2=8.0,
                 literal=False, k_range=None, n_threads=0):
    ic, j12, m12, _ = states
    P = ind.shape[0]
    nR = len(R)
    mat = np.zeros(P * nR)
    y2 = np.zeros(P * nR)
    sk = np.zeros(P, np.int32)
    k0, k1 = (0, P) if k_range is None else k_range
    g = Grid(*grid) if not isinstance(grid, Grid) else grid
    rc = lib().orc_build_matrix(C.byref(osys.s), len(ic), ic, j12, m12, P,
                                np.ascontiguousarray(ind, dtype=np.int32).reshape(-1), nR,
                                np.ascontiguousarray(R, dtype=np.float64), C.byref(g),
                                C.byref(pes.s), mij_cut, r_cut1, r_cut2, 1 if literal else 0,
                                k0, k1, n_threads, mat, y2, sk)
    if rc:
        raise RuntimeError(f"orc_build_matrix failed: {rc}")
    return mat.reshape(P, nR), y2.reshape(P, nR), sk


def integrate_elements(osys, states, ind, R, grid, pes, literal=False, k_range=None,
                       r_range=None, n_threads=0):
    ic, j12, m12, _ = states
    P = ind.shape[0]
    nR = len(R)
    mat = np.zeros(P * nR)
    k0, k1 = (0, P) if k_range is None else k_range
    r0, r1 = (0, nR) if r_range is None else r_range
    g = Grid(*grid) if not isinstance(grid, Grid) else grid
    rc = lib().orc_integrate_elements(C.byref(osys.s), len(ic), ic, j12, m12, P,
                                      np.ascontiguousarray(ind, dtype=np.int32).reshape(-1), nR,
                                      np.ascontiguousarray(R, dtype=np.float64), C.byref(g),
                                      C.byref(pes.s), 1 if literal else 0, k0, k1, r0, r1,
                                      n_threads, mat)
    if rc:
        raise RuntimeError(f"orc_integrate_elements failed: {rc}")
    return mat.reshape(P, nR)


def read_mtrx_dat(path, n_state_cols):
    L = lib()
    ct, nch, ns, nR = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    P = C.c_int64()
    rc = L.orc_read_mtrx_dat_header(path.encode(), C.byref(ct), C.byref(nch), C.byref(ns),
                                    C.byref(P), C.byref(nR))
    if rc:
        raise IOError(f"bad MTRX.DAT header {path}")
    st = np.zeros(ns.value * n_state_cols, np.int32)
    ind = np.zeros(2 * P.value, np.int32)
    R = np.zeros(nR.value)
    mat = np.zeros(P.value * nR.value)
    rc = L.orc_read_mtrx_dat(path.encode(), n_state_cols, st, ind, R, mat)
    if rc:
        raise IOError(f"bad MTRX.DAT body {path} ({rc})")
    return dict(coll_type=ct.value, n_channels=nch.value, states=st.reshape(ns.value, n_state_cols),
                ind_mat=ind.reshape(P.value, 2), R=R, mat=mat.reshape(P.value, nR.value))


class OracleTables:
    def __init__(self, j12, m12, ej_hartree, ind, R, mat, y2, mass_au):
        self.j12 = np.ascontiguousarray(j12, np.int32)
        self.m12 = np.ascontiguousarray(m12, np.int32)
        self.ej = np.ascontiguousarray(ej_hartree, np.float64)
        self.ind = np.ascontiguousarray(ind, np.int32).reshape(-1)
        self.R = np.ascontiguousarray(R, np.float64)
        self.mat = np.ascontiguousarray(mat, np.float64).reshape(-1)
        self.y2 = np.ascontiguousarray(y2, np.float64).reshape(-1)
        self.s = Tables(len(self.j12), _ptr(self.j12), _ptr(self.m12), _ptr(self.ej),
                        len(self.ind) // 2, _ptr(self.ind), len(self.R), _ptr(self.R),
                        _ptr(self.mat), _ptr(self.y2), mass_au)


def make_traj(e_coll, l_real, s_st, dt, r_start, r_fin, numb_orb=1, numb_oscl=1, time_lim=0.0,
              max_steps=0, method=0, eps=1e-6, hmin=0.0, cs=False):
    """method 0: RK4 with step dt; 1: adaptive Cash-Karp (ODEINT) with accuracy eps and
    minimum step hmin inside every interval dt.  cs: the coupled-states approximation
    (CS_APPROX = YES)."""
    return Traj(e_coll, l_real, s_st, dt, r_start, r_fin, numb_orb, numb_oscl, time_lim, max_steps,
                method, eps, hmin, 1 if cs else 0)


def propagate_batch(tables, trajs, n_threads=0):
    N = len(tables.j12)
    n = len(trajs)
    arr = (Traj * n)(*trajs)
    amp = np.zeros(n * 2 * N)
    cls = np.zeros(n * 6)
    diag = np.zeros(n * 8)
    lib().orc_propagate_batch(C.byref(tables.s), n, arr, n_threads, amp, cls, diag)
    return amp.reshape(n, 2 * N), cls.reshape(n, 6), diag.reshape(n, 8)


def dotraject_at(tables, traj, at_rec, ):
    N = len(tables.j12)
    rec = np.ascontiguousarray(at_rec, np.float64).reshape(-1)
    amp = np.zeros(2 * N)
    diag = np.zeros(8)
    lib().orc_dotraject_at(C.byref(tables.s), C.byref(traj), len(rec) // 8, rec, amp, diag)
    return amp, diag


def derivs(tables, t, q):
    dq = np.zeros_like(q)
    lib().orc_derivs(C.byref(tables.s), t, np.ascontiguousarray(q, np.float64), dq)
    return dq


def inelast(n_channels, j_ini, J_down, J_up, L_min, prob, k_vec, dl=1):
    sig = np.zeros(n_channels)
    p = np.ascontiguousarray(prob, np.float64)
    rc = lib().orc_inelast_dl(n_channels, j_ini, J_down, J_up, L_min, dl, p.shape[0],
                              p.reshape(-1), k_vec, sig)
    if rc:
        raise RuntimeError(f"orc_inelast_dl failed: {rc}")
    return sig


def dotraject_record(tables, traj, max_rec=1 << 20):
    """DOTRAJECT with SAVE_TRAJECT: (amp, cls, diag, records n x 8)."""
    N = len(tables.j12)
    amp = np.zeros(2 * N)
    cls = np.zeros(6)
    diag = np.zeros(8)
    rec = np.zeros(8 * max_rec)
    n = C.c_int64(0)
    lib().orc_dotraject_rec(C.byref(tables.s), C.byref(traj), amp, cls, diag, rec, max_rec,
                            C.byref(n))
    if n.value > max_rec:
        raise RuntimeError(f"{n.value} records exceed max_rec={max_rec}")
    return amp, cls, diag, rec[:8 * n.value].reshape(n.value, 8)


def expansion_matrix_type8(osys, states, ind, labels, terms):
    """SYS_TYPE 8 matrix (P x nR, Hartree) from PES expansion terms (nR x n_terms, cm^-1)."""
    ic, j12, m12, _ = states
    ind = np.ascontiguousarray(ind, np.int32)
    labels = np.ascontiguousarray(labels, np.int32)
    terms = np.ascontiguousarray(terms, np.float64)
    P, nR = ind.shape[0], terms.shape[0]
    mat = np.zeros(P * nR)
    rc = lib().orc_expansion_matrix_type8(C.byref(osys.s), _ptr(ic), _ptr(j12), _ptr(m12), P,
                                          _ptr(ind.reshape(-1)), labels.shape[0],
                                          _ptr(labels.reshape(-1)), nR, _ptr(terms), _ptr(mat))
    if rc:
        raise RuntimeError(f"orc_expansion_matrix_type8 failed: {rc}")
    return mat.reshape(P, nR)


def expansion_matrix_atom(osys, states, ind, labels, terms, e_unit):
    """SYS_TYPE 1, 3 or 4 matrix (P x nR, Hartree) from PES expansion terms (nR x n_terms in
    the unit e_unit Hartree); labels: one row per term, (l,) or (l, nju)."""
    ic, j12, m12, _ = states
    ind = np.ascontiguousarray(ind, np.int32)
    lab = np.asarray(labels, np.int32).reshape(len(labels), -1)
    a_top = np.zeros((len(lab), 5), np.int32)
    a_top[:, :lab.shape[1]] = lab
    terms = np.ascontiguousarray(terms, np.float64)
    P, nR = ind.shape[0], terms.shape[0]
    mat = np.zeros(P * nR)
    rc = lib().orc_expansion_matrix_atom(C.byref(osys.s), _ptr(ic), _ptr(j12), _ptr(m12), P,
                                         _ptr(ind.reshape(-1)), len(lab), _ptr(a_top.reshape(-1)),
                                         nR, _ptr(terms), e_unit, _ptr(mat))
    if rc:
        raise RuntimeError(f"orc_expansion_matrix_atom failed: {rc}")
    return mat.reshape(P, nR)


def expansion_matrix_type0(osys, states, ind, labels, terms, e_unit):
    """SYS_TYPE 0 matrix (P x nR, Hartree) from PES expansion terms (nR x n_terms, in the
    unit e_unit Hartree); labels n_terms x 5 (l1, nju1, l2, nju2, l)."""
    ic, j12, m12, _ = states
    ind = np.ascontiguousarray(ind, np.int32)
    labels = np.ascontiguousarray(labels, np.int32).reshape(-1, 5)
    terms = np.ascontiguousarray(terms, np.float64)
    P, nR = ind.shape[0], terms.shape[0]
    mat = np.zeros(P * nR)
    rc = lib().orc_expansion_matrix_type0(C.byref(osys.s), _ptr(ic), _ptr(j12), _ptr(m12), P,
                                          _ptr(ind.reshape(-1)), labels.shape[0],
                                          _ptr(labels.reshape(-1)), nR, _ptr(terms), e_unit,
                                          _ptr(mat))
    if rc:
        raise RuntimeError(f"orc_expansion_matrix_type0 failed: {rc}")
    return mat.reshape(P, nR)


def expansion_matrix_type7(osys, states, ind, labels, terms, e_unit):
    """SYS_TYPE 7 matrix (P x nR, Hartree) from PES expansion terms (nR x n_terms, in the
    unit e_unit Hartree); labels n_terms x 4 (l1, nju1, l2, l); the system's ka1 = k,
    kc1 = eps."""
    ic, j12, m12, _ = states
    ind = np.ascontiguousarray(ind, np.int32)
    labels = np.ascontiguousarray(labels, np.int32).reshape(-1, 4)
    terms = np.ascontiguousarray(terms, np.float64)
    P, nR = ind.shape[0], terms.shape[0]
    mat = np.zeros(P * nR)
    rc = lib().orc_expansion_matrix_type7(C.byref(osys.s), _ptr(ic), _ptr(j12), _ptr(m12), P,
                                          _ptr(ind.reshape(-1)), labels.shape[0],
                                          _ptr(labels.reshape(-1)), nR, _ptr(terms), e_unit,
                                          _ptr(mat))
    if rc:
        raise RuntimeError(f"orc_expansion_matrix_type7 failed: {rc}")
    return mat.reshape(P, nR)


def expansion_matrix_type0_identical(osys, states, parity, ind, labels, terms, e_unit):
    """SYS_TYPE 0 matrix for identical partners (P x nR, Hartree); parity: exchange parity
    per state; labels n_terms x 5."""
    ic, j12, m12, _ = states
    par = np.ascontiguousarray(parity, np.int32)
    ind = np.ascontiguousarray(ind, np.int32)
    labels = np.ascontiguousarray(labels, np.int32).reshape(-1, 5)
    terms = np.ascontiguousarray(terms, np.float64)
    P, nR = ind.shape[0], terms.shape[0]
    mat = np.zeros(P * nR)
    rc = lib().orc_expansion_matrix_type0_identical(
        C.byref(osys.s), _ptr(np.ascontiguousarray(ic, np.int32)),
        _ptr(np.ascontiguousarray(j12, np.int32)), _ptr(np.ascontiguousarray(m12, np.int32)),
        _ptr(par), P, _ptr(ind.reshape(-1)), labels.shape[0], _ptr(labels.reshape(-1)), nR,
        _ptr(terms), e_unit, _ptr(mat))
    if rc:
        raise RuntimeError(f"orc_expansion_matrix_type0_identical failed: {rc}")
    return mat.reshape(P, nR)


def expansion_term(sys_type, l, l1, l2, nju1, nju2, beta1, gamma1, alpha2, beta2, gamma2=0.0):
    r, i = C.c_double(), C.c_double()
    lib().orc_expansion_term(sys_type, l, l1, l2, nju1, nju2, beta1, gamma1, alpha2, beta2, gamma2,
                             C.byref(r), C.byref(i))
    return r.value, i.value


def project_terms_atom(sys_type, labels, V, eq_gamma=True):
    """CALC_EXPANSION_TERMS for SYS_TYPE 1 (V: nR x n_beta), 3 and 4 (V: nR x n_beta x
    n_gamma); labels (l,) or (l, nju).  Returns (terms, terms_im), n_terms x nR."""
    lab = np.asarray(labels, np.int32).reshape(len(labels), -1)
    a_top = np.zeros((len(lab), 5), np.int32)
    a_top[:, :lab.shape[1]] = lab
    V = np.ascontiguousarray(V, np.float64)
    nR, nb = V.shape[:2]
    ng = V.shape[2] if V.ndim == 3 else 1
    T = np.zeros(nR * len(lab))
    Ti = np.zeros(nR * len(lab))
    rc = lib().orc_project_terms_atom(sys_type, len(lab), _ptr(a_top.reshape(-1)), nb, ng,
                                      1 if eq_gamma else 0, nR, _ptr(V), _ptr(T), _ptr(Ti))
    if rc:
        raise RuntimeError(f"orc_project_terms_atom failed: {rc}")
    return T.reshape(len(lab), nR), Ti.reshape(len(lab), nR)


def project_terms(sys_type, labels, V, eq_gamma=True):
    """CALC_EXPANSION_TERMS for SYS_TYPE 7, 8 and 0.  labels: one row per term, (l1, nju1,
    l2, l) for 7 and 8 or (l1, nju1, l2, nju2, l) for 0; V: (nR, n_alpha2, n_beta1,
    n_beta2, n_gamma1[, n_gamma2]).  Returns (terms, terms_im), each n_terms x nR."""
    lab = np.asarray(labels, np.int32).reshape(len(labels), -1)
    a_top = np.zeros((len(lab), 5), np.int32)
    a_top[:, :lab.shape[1]] = lab
    V = np.ascontiguousarray(V, np.float64)
    nR, n2, n3, n4, n5 = V.shape[:5]
    n6 = V.shape[5] if V.ndim == 6 else 1
    T = np.zeros(nR * len(lab))
    Ti = np.zeros(nR * len(lab))
    lib().orc_project_terms(sys_type, len(lab), _ptr(a_top.reshape(-1)), n2, n3, n4, n5, n6,
                            1 if eq_gamma else 0, nR, _ptr(V), _ptr(T), _ptr(Ti))
    return T.reshape(len(lab), nR), Ti.reshape(len(lab), nR)
