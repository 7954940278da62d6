"""rs_primes_generate_noalloc: the allocation-free prime generator.

It must produce, through the C ABI, the same primes as rs_primes_generate
(the context-based generator with allocated buffers) on two calls in a row
that reuse its static device scratch, report the full count when the caller's
array is too small, and reject ranges wider than its scratch limit.  This
file is collected last so the set-up also runs after the other tests' device
work; it passes alone as well.
"""
import ctypes as C

import numpy as np
import pytest


def _call(rs, p0, p1, out, cap, count, stream):
    L = rs.lib()
    return L.rs_primes_generate_noalloc(p0, p1, out, cap, count, stream)


def test_rejects_range_wider_than_scratch(rs):
    L = rs.lib()
    dummy = C.c_void_p(16)   # never dereferenced: the width check comes first
    rc = L.rs_primes_generate_noalloc(1 << 40, (1 << 40) + rs.NOALLOC_MAX_WIDTH + 1, dummy, 1, dummy, None)
    assert rc == rs.RS_EARG
    assert str(rs.NOALLOC_MAX_WIDTH) in L.rs_last_error().decode()
    assert L.rs_primes_generate_noalloc(100, 100, dummy, 1, dummy, None) == rs.RS_EARG
    assert L.rs_primes_generate_noalloc(3, 1000, dummy, 1, None, None) == rs.RS_EARG


@pytest.mark.gpu
def test_two_calls_in_a_row_match_allocating_generator(rs, sieve):
    import torch
    W = rs.NOALLOC_MAX_WIDTH
    ranges = [((1 << 50) + 12345, (1 << 50) + 12345 + W),      # Miller-Rabin region, full width
              (3, W)]                                            # sieve-only region with the smallest primes
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    st = torch.cuda.Stream(dev)
    caps = [W // 2, W // 2]
    outs = [torch.empty(cap, dtype=torch.int64, device=dev) for cap in caps]
    counts = torch.zeros(2, dtype=torch.int32, device=dev)
    st.wait_stream(torch.cuda.current_stream(dev))
    for i, (a, b) in enumerate(ranges):
        rc = _call(rs, a, b, outs[i].data_ptr(), caps[i], counts.data_ptr() + 4 * i, st.cuda_stream)
        assert rc == rs.RS_OK, rs.lib().rs_last_error().decode()
    st.synchronize()
    n = counts.cpu().numpy().astype(np.int64)
    for i, (a, b) in enumerate(ranges):
        want = np.sort(sieve.primes(a, b))
        got = np.sort(outs[i][: n[i]].cpu().numpy().view(np.uint64))
        assert n[i] == len(want) > 0
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_small_output_reports_full_count(rs, sieve):
    import torch
    a, b = (1 << 44) + 1, (1 << 44) + 1 + 200_000
    want = np.sort(sieve.primes(a, b))
    dev = torch.device("cuda:0")
    st = torch.cuda.Stream(dev)
    cap = 1000
    out = torch.zeros(cap, dtype=torch.int64, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    st.wait_stream(torch.cuda.current_stream(dev))
    assert _call(rs, a, b, out.data_ptr(), cap, count.data_ptr(), st.cuda_stream) == rs.RS_OK
    st.synchronize()
    assert int(count.item()) == len(want) > cap
    # whatever was written is a true prime of the range, each at most once
    got = out.cpu().numpy().view(np.uint64)
    written = got[got != 0]
    assert np.isin(written, want).all()
    assert len(np.unique(written)) == len(written)
