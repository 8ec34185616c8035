"""adatm_gram_noalloc: the Gram entry point that allocates no device memory
(its partial sums live in a fixed device array), checked through the C ABI
against adatm_gram on the same rows, twice in a row."""
import ctypes as C

import pytest

import adatm_b200 as A

pytestmark = pytest.mark.gpu


def _rows(torch, rows, R, seed):
    ldr = (R + 3) // 4 * 4
    g = torch.Generator("cuda").manual_seed(seed)
    x = torch.rand(rows, ldr, device="cuda", dtype=torch.float32, generator=g) - 0.25
    x[:, R:] = 0
    return x, ldr


@pytest.mark.parametrize("rows,R", [(1, 1), (300, 16), (5000, 32), (20000, 64), (777, 50)])
def test_gram_noalloc_matches_gram(gpu, rows, R):
    import torch
    lib = A.lib()
    assert lib.adatm_set_device(0) == A.SPLATT_SUCCESS
    x, ldr = _rows(torch, rows, R, rows + R)
    ref = torch.zeros(R, R, device="cuda", dtype=torch.float64)
    assert lib.adatm_gram(C.c_void_p(x.data_ptr()), rows, R, ldr, C.c_void_p(ref.data_ptr())) \
        == A.SPLATT_SUCCESS, A._native.last_error()
    for _ in range(2):
        G = torch.full((R, R), float("nan"), device="cuda", dtype=torch.float64)
        rc = lib.adatm_gram_noalloc(C.c_void_p(x.data_ptr()), rows, R, ldr, C.c_void_p(G.data_ptr()), None)
        assert rc == A.SPLATT_SUCCESS, A._native.last_error()
        assert torch.allclose(G, ref, rtol=1e-12, atol=1e-12 * float(ref.abs().max()))


def test_gram_noalloc_allocates_nothing(gpu):
    """After a first call (set-up), further calls leave the device's free
    memory unchanged, and they still succeed while a torch tensor holds
    nearly all of it."""
    import torch
    lib = A.lib()
    x, ldr = _rows(torch, 20000, 32, 5)
    G = torch.zeros(32, 32, device="cuda", dtype=torch.float64)
    call = lambda: lib.adatm_gram_noalloc(C.c_void_p(x.data_ptr()), 20000, 32, ldr,
                                          C.c_void_p(G.data_ptr()), None)
    assert call() == A.SPLATT_SUCCESS, A._native.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert call() == A.SPLATT_SUCCESS
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    ref = G.clone()
    hog = torch.empty(max(0, free0 - (256 << 20)), dtype=torch.uint8, device="cuda")
    try:
        assert call() == A.SPLATT_SUCCESS, A._native.last_error()
        assert torch.equal(G, ref)
    finally:
        del hog
        torch.cuda.empty_cache()


def test_gram_noalloc_rejects_rank_above_scratch(gpu):
    import torch
    lib = A.lib()
    x, ldr = _rows(torch, 64, 65, 1)
    G = torch.zeros(65, 65, device="cuda", dtype=torch.float64)
    rc = lib.adatm_gram_noalloc(C.c_void_p(x.data_ptr()), 64, 65, ldr, C.c_void_p(G.data_ptr()), None)
    assert rc == A.SPLATT_ERROR_BADINPUT
    assert "64" in A._native.last_error()
