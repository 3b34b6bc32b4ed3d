"""Seeded synthetic potential energy surfaces and the benchmark configurations.

The reference plugs a fitted ab-initio surface into USER_DEFINED_PES
(PES_DIRECTORIES/*, called through MQCT_SOURCE_CODES/pes_sys_type.f).  The
workloads here use seeded synthetic surfaces of the shapes the benchmark
configurations state; every parameter is generated from a fixed seed so the
GPU build and the CPU oracle see identical inputs.
"""
from __future__ import annotations

import numpy as np

# PES kinds of the C ABI (MQCT_PES_* in include/mqct_b200.h).  Kept here as plain
# numbers so that this module also loads on its own, without the CUDA library (the
# CPU baseline builds its inputs from it).
PES_TABLE, PES_LEGENDRE, PES_SITES1, PES_SITES2 = 0, 1, 2, 3

AMU_TO_AU = 1822.8885          # MQCT_SOURCE_CODES/iotest.f:24
EV_TO_WN = 8065.5448
AU_TO_EV = 27.21113845
CM_TO_HARTREE = 1.0 / EV_TO_WN / AU_TO_EV
A_BOHR = 0.52917721067


def legendre_pes(n_lambda=7, seed=1):
    """V(R,theta) = sum_l [A_l e^{-b_l R} - C_l / R^6] P_l(cos theta), l = 0..n_lambda-1,
    A ~ U(1e3, 1e5) cm^-1, b ~ U(1.5, 2.5) bohr^-1, C ~ U(1e4, 1e5) cm^-1 bohr^6."""
    rng = np.random.default_rng(seed)
    A = rng.uniform(1e3, 1e5, n_lambda)
    b = rng.uniform(1.5, 2.5, n_lambda)
    Cc = rng.uniform(1e4, 1e5, n_lambda)
    return dict(kind=PES_LEGENDRE, n_terms=n_lambda, params=np.concatenate([A, b, Cc]),
                sites1=None, sites2=None)


# Three rigid sites of a bent triatomic in the rotor frame (x = a, y = b,
# z = c axis of the Hamiltonian of MQCT_SOURCE_CODES/asym_top.f:103-137), bohr.
TRIATOMIC_SITES = np.array([[0.0, -0.1241, 0.0],
                            [1.4309, 0.9849, 0.0],
                            [-1.4309, 0.9849, 0.0]])


def site_pes(n_terms=12, seed=2, sites=TRIATOMIC_SITES):
    """Rotor + atom site-site surface: n_terms Morse + damped dispersion terms
    spread over the sites, D ~ U(20, 200) cm^-1, a ~ U(0.8, 1.4) bohr^-1,
    r_e ~ U(5, 7) bohr, C6 ~ U(1e4, 1e5) cm^-1 bohr^6, damping radius r_d = r_e."""
    rng = np.random.default_rng(seed)
    n_sites = len(sites)
    p = np.zeros((n_terms, 6))
    p[:, 0] = np.arange(n_terms) % n_sites
    p[:, 1] = rng.uniform(20.0, 200.0, n_terms)
    p[:, 2] = rng.uniform(0.8, 1.4, n_terms)
    p[:, 3] = rng.uniform(5.0, 7.0, n_terms)
    p[:, 4] = rng.uniform(1e4, 1e5, n_terms)
    p[:, 5] = p[:, 3]
    return dict(kind=PES_SITES1, n_terms=n_terms, params=p.reshape(-1),
                sites1=np.ascontiguousarray(sites, dtype=np.float64).reshape(-1), sites2=None)


def rotor_sites9(seed=5, sites=TRIATOMIC_SITES):
    """Nine interaction sites of a rigid triatomic: its three atoms plus six seeded
    off-atom sites within 1.5 bohr of the centre of the atoms, bohr."""
    rng = np.random.default_rng(seed)
    extra = rng.uniform(-1.5, 1.5, (6, 3)) + np.mean(sites, axis=0)
    return np.concatenate([np.asarray(sites, np.float64), extra])


def site_pes2(seed=4, sites1=None, sites2=None):
    """Rotor + rotor site-site surface (SITES2): one Morse + damped-dispersion term
    per pair of sites (9 x 9 = 81 terms for the nine-site rotors), D ~ U(20, 200)/9
    cm^-1 (so the 81 terms add up to the depth of one rotor-atom well), a ~ U(0.8,
    1.4) bohr^-1, r_e ~ U(5, 7) bohr, C6 ~ U(1e4, 1e5)/9 cm^-1 bohr^6, r_d = r_e.
    Rotor 1 sits at the origin, rotor 2 at R along z."""
    s1 = rotor_sites9() if sites1 is None else np.asarray(sites1, np.float64)
    s2 = s1 if sites2 is None else np.asarray(sites2, np.float64)
    rng = np.random.default_rng(seed)
    n1, n2 = len(s1), len(s2)
    n = n1 * n2
    p = np.zeros((n, 7))
    p[:, 0] = np.repeat(np.arange(n1), n2)
    p[:, 1] = np.tile(np.arange(n2), n1)
    p[:, 2] = rng.uniform(20.0, 200.0, n) / 9.0
    p[:, 3] = rng.uniform(0.8, 1.4, n)
    p[:, 4] = rng.uniform(5.0, 7.0, n)
    p[:, 5] = rng.uniform(1e4, 1e5, n) / 9.0
    p[:, 6] = p[:, 4]
    return dict(kind=PES_SITES2, n_terms=n, params=p.reshape(-1),
                sites1=np.ascontiguousarray(s1).reshape(-1),
                sites2=np.ascontiguousarray(s2).reshape(-1))


def asym_channels(jmax):
    """(j, Ka, Kc) levels of an asymmetric top for j <= jmax in the JMIN/JMAX order
    (MQCT_SOURCE_CODES/iotest.f:6603-6617, labels of MQCT_SOURCE_CODES/asym_top.f:139-173)."""
    out = []
    for j in range(jmax + 1):
        ka = [0] + [i // 2 for i in range(2, 2 * j + 2)]
        kc = ka[::-1]
        out += [(j, ka[i], kc[i]) for i in range(2 * j + 1)]
    return out


# ---------------------------------------------------------------- configurations
def config_c1():
    """Rigid diatom (B = 1.93 cm^-1) + atom, j = 0..10 all m (121 states),
    Legendre PES, 64 GL theta points, 200 R points 3-20 bohr; 100 trajectories at
    E = 500 cm^-1, b uniform 0-12 bohr, RK4 dt = 10 a.u., initial j = 0."""
    return dict(name="c1_diatom_atom", sys_type=1, channels=[(j,) for j in range(11)],
                BE=1.93, grid=(64, 0, 0, 0, 0, 0, 1), nR=200, rmin=3.0, rmax=20.0,
                pes=legendre_pes(7, seed=1), mass_amu=3.5019, E_cm=500.0, b_max=12.0,
                n_traj=100, dt=10.0)


def config_c2(alpha_grid=True):
    """Asymmetric top (A, B, C = 27.9, 14.5, 9.3 cm^-1) + atom, j <= 8 all tau and m
    (81 levels, 969 states, 31 977 pairs), 12-term site-site PES, grid 48 GL beta x
    48 gamma (x 48 alpha as written), 300 R points 3-25 bohr."""
    # JMIN/JMAX channel generation: j ascending, tau = -j..j with the (Ka, Kc)
    # labels of STATE (MQCT_SOURCE_CODES/iotest.f:6603-6617,
    # MQCT_SOURCE_CODES/asym_top.f:139-173).
    chans = []
    for j in range(9):
        ka_list = [0] + [i // 2 for i in range(2, 2 * j + 2)]
        kc_list = ka_list[::-1]
        for i in range(2 * j + 1):
            chans.append((j, ka_list[i], kc_list[i]))
    return dict(name="c2_asym_top_atom", sys_type=4, channels=chans, A=27.9, B=14.5, C=9.3,
                grid=(48, 48, 48 if alpha_grid else 0, 0, 0, 0, 1), nR=300, rmin=3.0,
                rmax=25.0, pes=site_pes(12, seed=2), mass_amu=3.7523705333)


def config_c4(jmax=5, j12_sum_max=None, grid_n=24):
    """Two asymmetric tops (A, B, C = 27.9, 14.5, 9.3 cm^-1 each), channel pairs with
    j1, j2 <= jmax (and j1 + j2 <= j12_sum_max if given), 5-D grid grid_n^5 (GL in
    both beta, midpoint in alpha2, gamma1, gamma2), 200 R points 4-25 bohr, the 81-term
    SITES2 surface, reduced mass 9.00764 amu."""
    lv = asym_channels(jmax)
    chans = [(a + b) for a in lv for b in lv
             if j12_sum_max is None or a[0] + b[0] <= j12_sum_max]
    n = grid_n
    return dict(name="c4_two_asym_tops", sys_type=0, channels=chans, A=27.9, B=14.5, C=9.3,
                grid=(n, n, 0, n, n, n, 1), nR=200, rmin=4.0, rmax=25.0, pes=site_pes2(),
                mass_amu=9.00764)


def config_c3():
    """c2 matrix, 4096 trajectories, b ~ U(0, 15) bohr, E log-uniform 50-2000 cm^-1,
    RK4 dt = 5 a.u. until R > 25 bohr, FP32 amplitudes with FP64 phases."""
    rng = np.random.default_rng(3)
    n = 4096
    b = rng.uniform(0.0, 15.0, n)
    E = np.exp(rng.uniform(np.log(50.0), np.log(2000.0), n))
    return dict(name="c3_batched_propagation", n_traj=n, b=b, E_cm=E, dt=5.0, r_fin=25.0)
