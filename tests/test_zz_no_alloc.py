"""pxs_photometric_loss_static: the photometric loss with its scratch in a
static device array, for callers that cannot allocate device memory.

This file is collected last, so its GPU test also runs after every other test
has used the device; it passes run alone in a fresh process as well. The
outputs are checked against pxs_photometric_loss, one image at a time, on two
calls in a row with different batches (the second call finds the first
call's sums and image descriptors in the shared array)."""
import ctypes as ct

import numpy as np
import pytest

from parallax_b200 import _abi
from parallax_b200._lib import lib
import parallax_b200 as px

MAX_VIEWS = 64  # PXS_STATIC_LOSS_MAX_VIEWS


def _call(rendered, target, width, height, n_views, ssim_weight, dL, per_view, loss,
          stream=None):
    err = ct.create_string_buffer(256)
    status = lib().pxs_photometric_loss_static(rendered, target, width, height, n_views,
                                               ssim_weight, dL, per_view, loss, stream, err,
                                               len(err))
    return status, err.value.decode()


def test_rejects_more_views_than_the_static_scratch_holds():
    # argument checks come before any device call, so this needs no GPU
    status, why = _call(None, None, 8, 8, MAX_VIEWS + 1, 0.2, None, None, None)
    assert status == _abi.PXS_ERR_INVALID
    assert "limit of 64" in why
    status, why = _call(None, None, 8, 8, 2, 0.2, None, None, None)
    assert status == _abi.PXS_ERR_INVALID and "null" in why


@pytest.mark.gpu
def test_static_loss_matches_the_allocating_entry_point_twice():
    import torch
    torch.cuda.init()
    rng = np.random.default_rng(11)
    stream = torch.cuda.current_stream()
    for n_views, width, height, w in ((3, 67, 45, 0.2), (5, 40, 33, 0.5)):
        rendered = rng.random((n_views, height, width, 3), dtype=np.float32)
        target = np.clip(rendered + 0.1 * rng.standard_normal(rendered.shape,
                                                              dtype=np.float32), 0, 1)
        d_r = torch.from_numpy(rendered).cuda()
        d_t = torch.from_numpy(target).cuda()
        d_dL = torch.full_like(d_r, np.nan)
        d_per = torch.full((n_views,), np.nan, device="cuda")
        d_loss = torch.full((1,), np.nan, device="cuda")
        status, why = _call(d_r.data_ptr(), d_t.data_ptr(), width, height, n_views, w,
                            d_dL.data_ptr(), d_per.data_ptr(), d_loss.data_ptr(),
                            stream.cuda_stream)
        assert status == _abi.PXS_OK, why
        torch.cuda.synchronize()
        dL = d_dL.cpu().numpy()
        per = d_per.cpu().numpy()
        for v in range(n_views):
            o_loss, o_grad = px.photometric_loss(rendered[v], target[v], width, height, w)
            assert abs(per[v] - o_loss) <= 1e-5 * abs(o_loss)
            assert np.abs(dL[v] - o_grad).max() <= 1e-5 * np.abs(o_grad).max()
        expect = float(np.mean([px.photometric_loss(rendered[v], target[v], width, height, w,
                                                    want_gradient=False)[0]
                                for v in range(n_views)]))
        assert abs(float(d_loss.item()) - expect) <= 1e-5 * abs(expect)
