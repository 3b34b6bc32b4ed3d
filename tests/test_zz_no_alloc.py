"""GPU check of mqct_spline_y2_noalloc, the spline fit that allocates no device
memory: called twice in a row through the C ABI on device buffers, it returns
the spline second derivatives that mqct_build_matrix returns for the same
columns (same cut-off flags), the device's free memory does not change across a
call, the largest accepted grid (nR = 399) works, and a grid beyond that limit is
rejected."""
import numpy as np
import pytest

from mqct_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _system(mq):
    chans = [c for c in syn.config_c2()["channels"] if c[0] <= 2]
    return mq.CollisionSystem(4, chans, A=27.9, B=14.5, C=9.3)


def _check_calls(mq, R, mat, y2, sk, n_calls=2):
    import torch
    from mqct_b200 import _abi
    L = _abi.lib()
    P, nR = mat.shape
    dev = torch.device("cuda")
    d_R = torch.tensor(R, dtype=torch.float64, device=dev)
    d_mat = torch.tensor(mat, dtype=torch.float64, device=dev)
    d_sk = torch.tensor(sk.astype(np.int32), device=dev)
    outs = [torch.full((P, nR), float("nan"), dtype=torch.float64, device=dev)
            for _ in range(n_calls)]
    stream = torch.cuda.current_stream().cuda_stream
    scale = np.abs(y2).max()
    torch.cuda.synchronize()
    for i in range(n_calls):
        free0 = torch.cuda.mem_get_info()[0]
        _abi.check(L.mqct_spline_y2_noalloc(d_R.data_ptr(), nR, d_mat.data_ptr(), d_sk.data_ptr(),
                                            P, outs[i].data_ptr(), stream))
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if i > 0:  # the first call may load the library's device code on this device
            assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
        got = outs[i].cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - y2)) <= 1e-12 * scale
        assert np.all(got[sk.astype(bool)] == 0.0)


def test_noalloc_spline_matches_build_matrix(mq, gpu_available):
    s = _system(mq)
    R = mq.r_grid(120, 3.0, 25.0)
    mat, y2, sk = mq.build_matrix(s, R, (12, 12, 0, 0, 0, 0, 1), syn.site_pes(12, seed=2),
                                  precision=mq.PREC_FP64)
    assert sk.any() and not sk.all()  # some columns flagged by the cut-off
    _check_calls(mq, R, mat, y2, sk, n_calls=3)


def test_noalloc_spline_largest_grid(mq, gpu_available):
    s = _system(mq)
    R = mq.r_grid(399, 3.0, 25.0)
    mat, y2, sk = mq.build_matrix(s, R, (8, 8, 0, 0, 0, 0, 1), syn.site_pes(12, seed=2),
                                  precision=mq.PREC_FP64)
    assert sk.any() and not sk.all()
    _check_calls(mq, R, mat, y2, sk, n_calls=2)


def test_noalloc_spline_rejects_grid_beyond_limit(mq, gpu_available):
    import torch
    from mqct_b200 import _abi
    L = _abi.lib()
    nR = 400
    d_R = torch.linspace(3.0, 25.0, nR, dtype=torch.float64, device="cuda")
    d_mat = torch.zeros((2, nR), dtype=torch.float64, device="cuda")
    d_y2 = torch.zeros_like(d_mat)
    rc = L.mqct_spline_y2_noalloc(d_R.data_ptr(), nR, d_mat.data_ptr(), None, 2, d_y2.data_ptr(), None)
    assert rc == -5
    assert b"399" in L.mqct_last_error()
