"""The give-up paths of the library's bounded device waits, made to run out on
purpose through gsparc_set_wait_limit (no GPU fault, no hang: a wait that runs
out sets its error bit, the kernel drains its own tensor-core work, frees its
tensor memory and returns).

* depth sort (look-back and the cooperative launch's per-receiver barrier):
  with the limit at 0, the first wait that is not already satisfied gives up
  and kErrSortWait (bit 3) appears in the error word; later stages skip their
  work.
* BF16 tensor-core MLP (mbarrier waits on the MMAs): with the limit at 0 every
  wait gives up at once, so kErrMlpWait (bit 4) is set by the forward and by
  the adjoint.
After the limit is restored the next calls are clean and give the results of
calls made before the limit was set (bit for bit where the work is
deterministic; the adjoint's float atomics within 2e-3 of each tensor's peak,
as the BF16 tests state)."""
import ctypes

import numpy as np
import pytest
import torch

from gsparc_b200 import _lib, raster, scenes
from gsparc_b200.shared_mlp import SharedMLP

pytestmark = pytest.mark.gpu

ERR_SORT_WAIT, ERR_MLP_WAIT = 1 << 3, 1 << 4


def _status(st):
    K = ctypes.c_longlong(0)
    err = ctypes.c_uint(0)
    s = _lib.lib().gsparc_read_status(_lib.ptr(st.image), ctypes.byref(K), ctypes.byref(err),
                                      _lib.stream_of(st.image.device))
    return int(s), int(K.value), int(err.value)


def _scene(P, R, seed):
    dev = torch.device("cuda")
    sc = scenes.make_scene(P, seed=seed)
    rx = scenes.make_receivers(R)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    m, s, q, o = sc.activated()
    return dict(means=t(m), scales=t(s), rots=t(q), opac=t(o.reshape(-1)), mlp=t(sc.mlp),
                views=t(scenes.view_matrices(rx)), rxs=t(rx), tx=t(scenes.TX_POS))


def _render(sc, **kw):
    return raster.forward(sc["means"], kw.pop("mlp", sc["mlp"]), sc["opac"], sc["scales"], sc["rots"], 90, 360, 1.0,
                          sc["views"], sc["tx"], sc["rxs"], **kw)


def test_depth_sort_wait_gives_up_then_recovers():
    L = _lib.lib()
    sc = _scene(8192, 4, seed=3)     # four 2,048-key CTAs per receiver: the sort waits across CTAs
    out0, _, _, st0 = _render(sc)
    assert _status(st0)[0] == 0
    seen = False
    try:
        assert L.gsparc_set_wait_limit(0) == 0
        for _ in range(10):          # a wait already satisfied when first polled does not give up
            _, _, _, st = _render(sc)
            status, K, err = _status(st)
            assert err & ~ERR_SORT_WAIT == 0
            if err & ERR_SORT_WAIT:
                assert status == 4   # GSPARC_ERR_DEVICE
                seen = True
                break
    finally:
        L.gsparc_set_wait_limit(-1)
    assert seen
    out1, _, _, st1 = _render(sc)
    assert _status(st1) == (0, _status(st0)[1], 0)
    assert torch.equal(out0, out1)


def test_bf16_mlp_waits_give_up_then_recover():
    L = _lib.lib()
    P, R = 2999, 2
    sc = _scene(P, R, seed=7)
    mlp = SharedMLP(3, 128, "gelu", precision="bf16")
    params = mlp.init_params(seed=5)
    gen = torch.Generator().manual_seed(8)

    def fwd():
        _, _, radii, st = _render(sc, mlp=None, shared=mlp, shared_params=params)
        return radii, st

    def bwd(st, radii, dsig):
        dparams = torch.empty_like(params)
        dmeans = torch.zeros_like(sc["means"])
        mlp.backward(P, R, sc["means"], sc["rxs"], params, st.geom, dsig, dparams, dmeans, st.image)
        return dparams, dmeans

    radii, st = fwd()
    assert _status(st)[0] == 0
    sig0 = raster.state_views(st)["signal"].clone()
    dsig = (torch.randn((R, P, 2), generator=gen).cuda() * (radii > 0)[..., None]).contiguous()
    dp0, dm0 = bwd(st, radii, dsig)
    assert _status(st)[0] == 0
    try:
        assert L.gsparc_set_wait_limit(0) == 0
        _, st_f = fwd()
        assert _status(st_f)[2] & ERR_MLP_WAIT
    finally:
        L.gsparc_set_wait_limit(-1)
    # the adjoint's give-up: a clean forward, then the adjoint with the limit at 0
    radii, st = fwd()
    assert _status(st)[0] == 0
    try:
        L.gsparc_set_wait_limit(0)
        bwd(st, radii, dsig)
        assert _status(st)[2] & ERR_MLP_WAIT
    finally:
        L.gsparc_set_wait_limit(-1)
    # restored: clean and equal to the calls before
    radii, st = fwd()
    assert _status(st)[0] == 0
    vis = radii > 0      # culled pairs' signal entries are never written
    assert torch.equal(raster.state_views(st)["signal"][vis], sig0[vis])
    dp1, dm1 = bwd(st, radii, dsig)
    assert _status(st)[0] == 0
    for a, b in ((dp1, dp0), (dm1, dm0)):
        assert (a - b).abs().max().item() <= 2e-3 * b.abs().max().item() + 1e-7
