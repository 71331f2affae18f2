"""mm_scaled_abs_max_noalloc (scratch in the library's static device memory) against
mm_scaled_abs_max (scratch it allocates itself), both through the C ABI.  The file is named to be
collected last, so that it also runs after every other GPU test has used the library."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT = 65536 * 4096  # cells: 65536 partial maxima of 4096 cells each
INVALID_ARGUMENT = 1  # mm_status MM_ERR_INVALID_ARGUMENT


@pytest.fixture(scope="module")
def L():
    from micromagnum_b200 import _lib
    return _lib


def field(n, prec, seed, zero_every=0, scale_to=1.0):
    dt = torch.float64 if prec == "f64" else torch.float32
    g = torch.Generator(device="cuda").manual_seed(seed)
    M = torch.randn(3 * n, generator=g, device="cuda", dtype=dt) * scale_to
    s = torch.rand(n, generator=g, device="cuda", dtype=dt) + 0.5
    if zero_every:
        s[::zero_every] = 0.0
    return M, s


def both(L, prec, M, s):
    p = L.MM_F64 if prec == "f64" else L.MM_F32
    n = s.numel()
    a, b = ctypes.c_double(), ctypes.c_double()
    L.check(L.lib().mm_scaled_abs_max(p, n, M.data_ptr(), s.data_ptr(), ctypes.byref(a), None))
    L.check(L.lib().mm_scaled_abs_max_noalloc(p, n, M.data_ptr(), s.data_ptr(), ctypes.byref(b), None))
    return a.value, b.value


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_matches_allocating_entry_point_twice_in_a_row(L, prec):
    # two calls in a row, the second smaller and with smaller values, so that partial maxima
    # left in the static scratch by the first call would show up in the second result
    M1, s1 = field(3_000_017, prec, 5, zero_every=7, scale_to=4e5)
    M2, s2 = field(70_001, prec, 6, scale_to=1e3)
    r = [both(L, prec, M1, s1), both(L, prec, M2, s2)]
    for ref, got in r:
        # the two kernels evaluate the same per-cell expression in double precision and the
        # maximum is exact, so the results agree to within one rounding of the final sqrt
        assert got == pytest.approx(ref, rel=4e-16, abs=0.0)
    assert r[1][1] < r[0][1]


@pytest.mark.parametrize("n", [1, 31, 4095, 4096, 4097, 65 * 4096 + 3])
def test_noalloc_sizes(L, n):
    M, s = field(n, "f64", n, zero_every=3 if n > 3 else 0)
    ref, got = both(L, "f64", M, s)
    assert got == pytest.approx(ref, rel=4e-16, abs=0.0)


def test_noalloc_all_scales_zero(L):
    M, s = field(10_000, "f32", 9)
    s.zero_()
    assert both(L, "f32", M, s) == (0.0, 0.0)


def test_noalloc_rejects_sizes_beyond_its_scratch(L):
    # real buffers of LIMIT + 1 cells (f32: 4.3 GB), so that every call here stays in bounds
    n = LIMIT + 1
    g = torch.Generator(device="cuda").manual_seed(13)
    M = torch.randn(3 * n, generator=g, device="cuda", dtype=torch.float32)
    s = torch.ones(n, device="cuda", dtype=torch.float32)
    out = ctypes.c_double()
    st = L.lib().mm_scaled_abs_max_noalloc(L.MM_F32, n, M.data_ptr(), s.data_ptr(), ctypes.byref(out), None)
    assert st == INVALID_ARGUMENT
    assert "exceeds its limit of 268435456 cells" in L.lib().mm_last_error().decode()
    # a field of exactly LIMIT cells (65536 full partials) is accepted (SoA stride LIMIT)
    a, b = ctypes.c_double(), ctypes.c_double()
    L.check(L.lib().mm_scaled_abs_max(L.MM_F32, LIMIT, M.data_ptr(), s.data_ptr(), ctypes.byref(a), None))
    L.check(L.lib().mm_scaled_abs_max_noalloc(L.MM_F32, LIMIT, M.data_ptr(), s.data_ptr(), ctypes.byref(b),
                                              None))
    assert b.value == pytest.approx(a.value, rel=4e-16, abs=0.0)
    del M, s
    torch.cuda.empty_cache()
