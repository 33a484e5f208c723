"""rsw_fft_forward_noalloc: the forward FFT for callers that cannot allocate
device memory (a process whose free device memory belongs to another
allocator, or a loop that must not pay cudaFree's device-wide sync).

The entry point keeps its scratch in a fixed array inside the library's
device image instead of allocating. This test calls it through the C ABI and
checks that it returns the same spectrum as the plan-based rsw_fft_forward
(within the FFT tolerance of the other GPU tests) on two calls in a row, that
it rejects lengths above its limit, and that a call leaves the device's free
memory unchanged. It runs alone in a fresh process as well as after the other
tests (its file name makes pytest collect it last)."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from rave_sim_b200 import _lib as L  # noqa: E402

TOL = {L.RSW_C128: 1e-12, L.RSW_C64: 2e-6}


def _field(n, seed, code):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    a = a.astype(np.complex128 if code == L.RSW_C128 else np.complex64)
    return torch.from_numpy(a).cuda()


def _rel(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _plan_fft(lib, x, code):
    plan = C.c_void_p()
    L.check(lib.rsw_plan_create(C.byref(plan), x.numel(), code))
    try:
        out = torch.empty_like(x)
        L.check(lib.rsw_fft_forward(plan, x.data_ptr(), out.data_ptr(), torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        return out
    finally:
        lib.rsw_plan_destroy(plan)


@pytest.mark.parametrize("code", [L.RSW_C128, L.RSW_C64])
@pytest.mark.parametrize("n", [1 << 10, 1 << 16])
def test_noalloc_matches_plan_fft_twice(n, code):
    lib = L.load()
    stream = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((1, 2)):  # two calls in a row share the scratch array
        x = _field(n, seed + 10 * n, code)
        ref = _plan_fft(lib, x, code)
        out = torch.empty_like(x)
        st = lib.rsw_fft_forward_noalloc(x.data_ptr(), out.data_ptr(), n, code, stream)
        assert st == L.RSW_OK, lib.rsw_last_error()
        torch.cuda.synchronize()
        assert _rel(out, ref) < TOL[code], f"call {call}"


def test_noalloc_in_place_and_alternating_lengths():
    lib = L.load()
    stream = torch.cuda.current_stream().cuda_stream
    for n, code in [(1 << 14, L.RSW_C128), (1 << 12, L.RSW_C64), (1 << 14, L.RSW_C128)]:
        x = _field(n, n, code)
        ref = _plan_fft(lib, x, code)
        y = x.clone()
        assert lib.rsw_fft_forward_noalloc(y.data_ptr(), y.data_ptr(), n, code, stream) == L.RSW_OK
        torch.cuda.synchronize()
        assert _rel(y, ref) < TOL[code]


def test_noalloc_rejects_sizes_beyond_limit():
    lib = L.load()
    x = torch.zeros(1 << 17, dtype=torch.complex128, device="cuda")
    st = lib.rsw_fft_forward_noalloc(x.data_ptr(), x.data_ptr(), 1 << 17, L.RSW_C128, None)
    assert st == L.RSW_ERR_INVALID
    assert b"no-allocation limit" in lib.rsw_last_error()
    assert lib.rsw_fft_forward_noalloc(x.data_ptr(), x.data_ptr(), 1000, L.RSW_C128, None) == L.RSW_ERR_INVALID


def test_noalloc_call_leaves_free_memory_unchanged():
    lib = L.load()
    n, code = 1 << 16, L.RSW_C128
    x = _field(n, 7, code)
    out = torch.empty_like(x)
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.rsw_fft_forward_noalloc(x.data_ptr(), out.data_ptr(), n, code, stream) == L.RSW_OK
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    assert lib.rsw_fft_forward_noalloc(x.data_ptr(), out.data_ptr(), n, code, stream) == L.RSW_OK
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_lengths_keep_their_own_tables():
    # each length and dtype has its own tables: alternating lengths, then
    # coming back to the first one, gives the plan's spectrum every time
    lib = L.load()
    stream = torch.cuda.current_stream().cuda_stream
    for i, (n, code) in enumerate([(1 << 10, L.RSW_C64), (1 << 12, L.RSW_C64), (1 << 10, L.RSW_C64),
                                   (1 << 15, L.RSW_C128), (1 << 12, L.RSW_C64), (1 << 10, L.RSW_C64)]):
        x = _field(n, 100 + i, code)
        ref = _plan_fft(lib, x, code)
        out = torch.empty_like(x)
        assert lib.rsw_fft_forward_noalloc(x.data_ptr(), out.data_ptr(), n, code, stream) == L.RSW_OK
        torch.cuda.synchronize()
        assert _rel(out, ref) < TOL[code], f"call {i}: n={n}"


def test_noalloc_first_call_for_a_length_refused_while_capturing():
    # the first call for a length and dtype builds its tables, which a graph
    # capture would only record: refused with RSW_ERR_INVALID, nothing launched
    lib = L.load()
    n, code = 1 << 5, L.RSW_C128  # a length no other test uses
    x = _field(n, 3, code)
    out = torch.empty_like(x)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        g.capture_begin()
        st = lib.rsw_fft_forward_noalloc(x.data_ptr(), out.data_ptr(), n, code, s.cuda_stream)
        torch.mul(x, 1.0, out=out)  # keep the graph non-empty
        g.capture_end()
    assert st == L.RSW_ERR_INVALID
    assert b"capturing" in lib.rsw_last_error()
    del g
    # outside the capture the same call builds the tables and succeeds
    ref = _plan_fft(lib, x, code)
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.rsw_fft_forward_noalloc(x.data_ptr(), out.data_ptr(), n, code, stream) == L.RSW_OK
    torch.cuda.synchronize()
    assert _rel(out, ref) < TOL[code]
