"""binius_fri_fold_codeword_noalloc: the allocation-free form of binius_fri_fold_codeword.

Some callers may not allocate device memory, or may not let a library allocate behind them: a
serving loop that admits prove requests by the free HBM it has budgeted for them, or a host that
hands the library slices of its own pre-allocated arena.  For them the library offers a fold entry
point whose intermediate buffer is a fixed 4 MiB static device array.  These tests call it through
the C ABI and require bit-identical output to the allocating entry point on two calls in a row (the
second call must not see anything left in the shared scratch by the first), plus a clear error when
the fold needs more scratch than the array holds.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU containers
    pytest.skip("needs a CUDA device", allow_module_level=True)

import binius64_b200 as bg  # noqa: E402
from binius64_b200 import _ffi  # noqa: E402


def _challenges(rng, n):
    arr = rng.integers(0, np.iinfo(np.uint64).max, size=(max(n, 1), 2), dtype=np.uint64,
                       endpoint=True)
    return arr


def _fold(entry, ntt, cw, log_len, ch, n):
    out = torch.empty((1 << (log_len - n), 2), dtype=torch.int64, device=cw.device)
    rc = entry(ntt.handle, cw.data_ptr(), log_len, ch.ctypes.data_as(ctypes.c_void_p), n,
               out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return rc, out


def test_noalloc_fold_matches_allocating_fold_twice():
    L = _ffi.lib()
    rng = np.random.default_rng(77)
    ntt = bg.AdditiveNTT(22)
    gen = torch.Generator(device="cuda").manual_seed(77)
    # Two calls in a row with different shapes and data; the second uses the whole scratch array
    # (log_len 22, 8 challenges -> 2^18 intermediate elements).
    for log_len, n in [(16, 6), (22, 8), (12, 3)]:
        cw = torch.randint(-2**63, 2**63 - 1, (1 << log_len, 2), dtype=torch.int64, device="cuda",
                           generator=gen)
        ch = _challenges(rng, n)
        rc_ref, ref = _fold(L.binius_fri_fold_codeword, ntt, cw, log_len, ch, n)
        _ffi.check(rc_ref)
        rc, got = _fold(L.binius_fri_fold_codeword_noalloc, ntt, cw, log_len, ch, n)
        _ffi.check(rc)
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (log_len, n)


def test_noalloc_fold_rejects_oversized_scratch():
    L = _ffi.lib()
    ntt = bg.AdditiveNTT(23)
    cw = torch.zeros((1 << 23, 2), dtype=torch.int64, device="cuda")
    ch = _challenges(np.random.default_rng(1), 5)
    before = L.binius_launch_count()
    rc, _ = _fold(L.binius_fri_fold_codeword_noalloc, ntt, cw, 23, ch, 5)
    assert rc == _ffi.BINIUS_E_ARG
    assert b"scratch" in L.binius_last_error()
    assert L.binius_launch_count() == before
