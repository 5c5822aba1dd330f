"""pf5d_abs_max_noalloc: the max-|a| reduction for callers that cannot let
the library allocate device memory (their own pool owns the GPU, or the loop
must never pay for cudaMalloc/cudaFree).  It must give exactly what
pf5d_abs_max gives -- a maximum is exact, so the tolerance is zero, as in
the other abs_max tests -- on consecutive calls that share its static
scratch, and it must refuse inputs larger than that scratch covers.

Kept in its own file, collected last, so a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from phasefield5d_b200 import _lib
    return torch, _lib, _lib.load()


def _both(cuda, a):
    torch, _lib, L = cuda
    res = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    s = _lib.stream_handle()
    _lib.check(L.pf5d_abs_max(_lib.ptr(a), a.numel(), ctypes_ptr(res, 0), s))
    _lib.check(L.pf5d_abs_max_noalloc(_lib.ptr(a), a.numel(), ctypes_ptr(res, 1), s))
    torch.cuda.synchronize()
    return res.cpu().numpy()


def ctypes_ptr(t, i):
    import ctypes
    return ctypes.c_void_p(t.data_ptr() + i * t.element_size())


def test_noalloc_matches_abs_max_on_two_calls(cuda):
    torch = cuda[0]
    rng = np.random.default_rng(42)
    big = rng.normal(size=3_000_017) * 3.0
    big[12345] = -97.25                      # the maximum, negative sign
    big[777] = np.nan                        # ignored by both
    small = rng.normal(size=10_001)          # second call: smaller input, smaller max
    for host in (big, small):
        a = torch.from_numpy(host).cuda()
        ref, got = _both(cuda, a)
        assert got == ref
        assert ref == np.nanmax(np.abs(host))


def test_noalloc_empty_and_limit(cuda):
    torch, _lib, L = cuda
    a = torch.zeros(0, dtype=torch.float64, device="cuda")
    ref, got = _both(cuda, a)
    assert got == ref == 0.0
    # The size check runs before anything is launched, so a one-element
    # buffer is enough to see the refusal.
    one = torch.zeros(1, dtype=torch.float64, device="cuda")
    res = torch.zeros(1, dtype=torch.float64, device="cuda")
    too_many = 32768 * 2048 + 1
    with pytest.raises(RuntimeError, match="at most"):
        _lib.check(L.pf5d_abs_max_noalloc(_lib.ptr(one), too_many, _lib.ptr(res),
                                          _lib.stream_handle()))


def test_noalloc_full_blocks_and_largest_size(cuda):
    """n an exact multiple of the 2048-element block (the last block full) and
    the largest n the scratch covers (32768 blocks: 512 MiB of doubles)."""
    torch = cuda[0]
    gen = torch.Generator(device="cuda").manual_seed(7)
    for n in (2048, 2048 * 37, 32768 * 2048):
        a = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
        a[n - 1] = -1e3                          # the maximum sits in the last, full block
        ref, got = _both(cuda, a)
        assert got == ref == 1e3
        del a
        torch.cuda.empty_cache()


_FRESH = r"""
import sys
sys.path.insert(0, {repo!r})
import torch
from phasefield5d_b200 import _lib
L = _lib.load()
a = torch.randn(1_000_003, dtype=torch.float64, device="cuda")
res = torch.zeros(1, dtype=torch.float64, device="cuda")
# one call on one element: the CUDA runtime's one-time set-up of the
# library's code on this context happens here
_lib.check(L.pf5d_abs_max_noalloc(_lib.ptr(a), 1, _lib.ptr(res), _lib.stream_handle()))
torch.cuda.synchronize()
free = [torch.cuda.mem_get_info()[0]]
for _ in range(2):
    _lib.check(L.pf5d_abs_max_noalloc(_lib.ptr(a), a.numel(), _lib.ptr(res),
                                      _lib.stream_handle()))
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
print(*free, res.item(), a.abs().max().item())
"""


def test_noalloc_first_call_leaves_device_memory_untouched(cuda):
    """In a fresh process (modules loaded eagerly), the first two calls on a
    million-element input leave the device's free memory exactly as it was,
    and the result is right.  The process first makes one call on a single
    element: the first launch into the library on a context lets the CUDA
    runtime set up the library's code there, which was seen to take 8 MiB
    of device memory once per process -- the runtime's doing, not an
    allocation by the entry point, whose scratch is the static array."""
    import os
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    out = subprocess.run([sys.executable, "-c", _FRESH.format(repo=repo)], env=env,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    f0, f1, f2, got, want = out.stdout.split()[-5:]
    assert int(f0) == int(f1) == int(f2), (f0, f1, f2)
    assert float(got) == float(want)
