"""GPU checks of the learned PES surrogate.

* the backward pass of the library's own kernels (loss and every parameter
  gradient) against a float64 torch reference of the same network on the same
  parameters and batch;
* training on seeded samples of the PES lowers the held-out error, and the
  trained network predicts the surface that the oracle evaluates;
* the matrix build with the surrogate: with a residual bound no check can meet,
  every radial point is re-evaluated exactly and the build equals the exact-PES
  build; with a working bound the elements stay close to the exact ones and the
  re-evaluations are counted.
"""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _torch_loss_grad(p, dims, X, y):
    import torch
    ts, off = [], 0
    for l in range(len(dims) - 1):
        n_w = dims[l] * dims[l + 1]
        W = torch.tensor(p[off:off + n_w].reshape(dims[l], dims[l + 1]), dtype=torch.float64,
                         requires_grad=True)
        off += n_w
        b = torch.tensor(p[off:off + dims[l + 1]], dtype=torch.float64, requires_grad=True)
        off += dims[l + 1]
        ts += [W, b]
    h = torch.tensor(X, dtype=torch.float64)
    for l in range(len(dims) - 1):
        z = h @ ts[2 * l] + ts[2 * l + 1]
        h = torch.nn.functional.silu(z) if l < len(dims) - 2 else z
    loss = ((h[:, 0] - torch.tensor(y, dtype=torch.float64)) ** 2).mean()
    loss.backward()
    return float(loss.detach()), np.concatenate([t.grad.numpy().reshape(-1) for t in ts])


def test_backward_matches_torch_reference(mq, gpu_available):
    sur = mq.Surrogate(4, syn.site_pes(12, seed=2), hidden=48, layers=3, seed=5)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((300, 11)).astype(np.float32)
    y = rng.standard_normal(300).astype(np.float32)
    loss, g = sur.loss_grad(X, y)
    loss_ref, g_ref = _torch_loss_grad(sur.params().astype(np.float64), [11, 48, 48, 48, 1], X, y)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    assert np.max(np.abs(g - g_ref)) <= 1e-4 * np.max(np.abs(g_ref))
    sur.close()


@pytest.fixture(scope="module")
def trained(mq):
    pes = syn.site_pes(12, seed=2)
    sur = mq.Surrogate(4, pes, hidden=128, layers=3, seed=3, r_min=3.0, r_max=20.0)
    loss, val = sur.train(n_samples=262144, epochs=12, batch=1024, lr=2e-3)
    yield sur, pes, loss, val
    sur.close()


def test_training_lowers_error_and_predicts_the_surface(mq, oracle, gpu_available, trained):
    sur, pes, loss, val = trained
    # asinh(V / 100 cm^-1) / 4 units; the 12-term wall keeps a network of this size
    # (and this training budget) near 0.07 -- a float64 torch run of the same
    # network and data reaches the same level
    assert loss[-1] < 0.2 * loss[0]
    assert val < 0.1, val
    rng = np.random.default_rng(7)
    n = 2000
    args = np.zeros((n, 6))
    args[:, 0] = rng.uniform(3.0, 20.0, n)
    args[:, 1] = rng.uniform(0.0, np.pi, n)
    args[:, 2] = rng.uniform(0.0, 2 * np.pi, n)
    v = sur.predict(args)
    opes = oracle.OraclePes(pes["kind"], pes["n_terms"], pes["params"], sites1=pes["sites1"])
    # the atom + rotor surface takes (-beta, -gamma) (pes_sys_type.f:36)
    ref = np.array([opes(a[0], 0.0, -a[1], -a[2]) for a in args])
    big = np.abs(ref) > 10.0
    rel = np.abs(v[big] - ref[big]) / np.abs(ref[big])
    assert np.median(rel) < 0.3, np.median(rel)


def _small_system(mq):
    chans = [c for c in syn.config_c2()["channels"] if c[0] <= 2]
    return mq.CollisionSystem(4, chans, A=27.9, B=14.5, C=9.3)


def test_matrix_build_with_surrogate(mq, gpu_available, trained):
    import torch
    sur, pes, _, _ = trained
    s = _small_system(mq)
    R = mq.r_grid(24, 4.0, 20.0)
    grid = (12, 12, 0, 0, 0, 0, 1)
    m0, _, _ = mq.build_matrix(s, R, grid, pes, precision=mq.PREC_FP64, mij_cutoff=0.0)
    n = s.P * len(R)
    dm = torch.empty(n, dtype=torch.float64, device="cuda")
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    dk = torch.empty(s.P, dtype=torch.int32, device="cuda")
    plan = mq.MatrixPlan(s, R, grid, pes, precision=mq.PREC_FP64, mij_cutoff=0.0)
    # a bound no check can meet: every radial point falls back to the exact surface
    plan.set_surrogate(sur, rel_bound=0.0, abs_bound_cm=1e-12, n_check=16)
    plan.execute(dm.data_ptr(), dy.data_ptr(), dk.data_ptr())
    plan.sync()
    n_exact, ratio = plan.surrogate_stats()
    assert n_exact == len(R) and ratio > 1.0
    m = dm.view(s.P, len(R)).cpu().numpy()
    assert np.max(np.abs(m - m0)) <= 1e-13 * np.abs(m0).max()
    # a working bound: the network serves the radial points it fits
    plan.set_surrogate(sur, rel_bound=0.2, abs_bound_cm=2.0, n_check=64)
    plan.execute(dm.data_ptr(), dy.data_ptr(), dk.data_ptr())
    plan.sync()
    n_exact, ratio = plan.surrogate_stats()
    assert 0 <= n_exact < len(R)
    m = dm.view(s.P, len(R)).cpu().numpy()
    rowmax = np.abs(m0).max(axis=1)
    sig = rowmax >= 1e-6 * rowmax.max()
    ek = np.abs(m - m0).max(axis=1)[sig] / rowmax[sig]
    # element errors follow the residual bound the network was held to
    assert np.median(ek) < 0.2 and ek.max() < 1.0, (np.median(ek), ek.max())
    plan.set_surrogate(None)
    plan.close()
