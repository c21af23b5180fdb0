"""GPU: the allocation-free readout (lnt_canonicalize_noalloc) against lnt_get_digits.

Some callers cannot allocate device memory when they need a residue in the
reference's digit format: a serving process that has handed all of its HBM to
its own pool or admission budget, a latency-critical step that must not pay
cudaMalloc's implicit device synchronisation, a checkpoint written by a path
that must not allocate.  They pass their own device buffers to
lnt_canonicalize_noalloc, whose scratch is one fixed library-owned array
(residues up to 2^24 words).  Its digits must equal the regular readout's
exactly (integer digits: the tolerance is zero), on two calls in a row that
share that array; up to the 2^24 limit they must equal canonical digits that
the test chose itself, rebuilt from perturbed balanced words.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc():
    from cuda_b200 import api

    f = api.lib().lnt_canonicalize_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _readout_twice(lnt, q, n, prp, first, second, start=None):
    """Two calls in a row through the no-alloc entry point, each checked
    against the regular readout of the same residue."""
    import torch

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn = _noalloc()
    with lnt.LucasTest(q, n, prp) as T:
        assert T.plan.startswith("RESIDENT")  # no pending run carries: raw words are the residue
        if start is not None:
            T.set_digits(start)
        widths = torch.from_numpy(T.widths()).to(dev)
        out = torch.empty(n, dtype=torch.int64, device=dev)
        for k in (first, second):
            T.iterate(k)
            expected = T.digits()
            words = torch.from_numpy(T.raw_state()).to(dev)
            out.fill_(-1)  # the readout must write every digit
            status = fn(words.data_ptr(), widths.data_ptr(), n, int(prp), 0, out.data_ptr(), stream)
            assert status == 0, lnt.lib().lnt_last_error()
            torch.cuda.synchronize(dev)
            got = out.cpu().numpy().view(np.uint64)
            assert np.array_equal(got, expected), (k, got[:4], expected[:4])


@pytest.mark.parametrize("q,n,prp", [(44497, 2048, False), (44497, 4096, True), (9973, 512, False),
                                     (1009, 64, True), (89, 4, False)])
def test_noalloc_matches_regular_readout(lnt, q, n, prp):
    _readout_twice(lnt, q, n, prp, 5, 17)


def test_noalloc_zero_residues(lnt):
    """Full tests of a Mersenne prime end on 0 (LL) and 9 (PRP); a PRP residue
    that starts at M (all digits maximal) stays M."""
    _readout_twice(lnt, 127, 8, False, 125, 1)  # LL: 0, then 0^2 - 2
    _readout_twice(lnt, 127, 8, True, 127, 3)
    from oracle import bigint_model as B

    full = np.array([(1 << w) - 1 for w in B.widths(127, 8)], dtype=np.uint64)
    _readout_twice(lnt, 127, 8, True, 1, 2, start=full)


def test_noalloc_rejects_sizes_beyond_its_scratch(lnt):
    import torch

    fn = _noalloc()
    dummy = torch.empty(8, dtype=torch.int64, device="cuda")
    for n in (1 << 25, 3, 0):
        assert fn(dummy.data_ptr(), dummy.data_ptr(), n, 0, 0, dummy.data_ptr(), None) == 1
    assert fn(None, dummy.data_ptr(), 8, 0, 0, dummy.data_ptr(), None) == 1
    assert b"2^24" in lnt.lib().lnt_last_error() or b"null" in lnt.lib().lnt_last_error()


def _balanced_words(rng, widths):
    """Random canonical digits d (value below M, not all maximal) and signed
    words of the same value: each digit above half its range borrows 2^w from
    the next word (cyclically: 2^q = 1 mod M), then random multiples of 2^w move
    between neighbours."""
    w = widths.astype(np.int64)
    d = (rng.integers(0, 1 << 62, size=w.size, dtype=np.int64) & ((np.int64(1) << w) - 1))
    d[-1] = 0  # not all maximal
    c = (d >= (np.int64(1) << (w - 1))).astype(np.int64)
    b = d - (c << w) + np.roll(c, 1)
    k = rng.integers(-3, 4, size=w.size, dtype=np.int64)
    b = b - (k << w) + np.roll(k, 1)
    return d.astype(np.uint64), b


@pytest.mark.parametrize("q,log2n", [(1000003, 16), (20000003, 20), (300000007, 24)])
def test_noalloc_at_size_limit(lnt, q, log2n):
    """n = 2^16, 2^20 and the declared limit 2^24 (262,144 scan blocks, the
    whole scratch array): two calls in a row, each digit equal to the
    canonical digits the words were built from."""
    import torch

    n = 1 << log2n
    assert lnt.secured_log2_length(q) == log2n
    dev = torch.device("cuda", 0)
    fn = _noalloc()
    with lnt.LucasTest(q, n, False) as T:
        widths_host = T.widths()
    widths = torch.from_numpy(widths_host).to(dev)
    out = torch.empty(n, dtype=torch.int64, device=dev)
    rng = np.random.default_rng(q)
    for _ in range(2):
        want, words_host = _balanced_words(rng, widths_host)
        words = torch.from_numpy(words_host).to(dev)
        out.fill_(-1)
        stream = torch.cuda.current_stream(dev)
        status = fn(words.data_ptr(), widths.data_ptr(), n, 0, 0, out.data_ptr(), stream.cuda_stream)
        assert status == 0, lnt.lib().lnt_last_error()
        got = out.cpu().numpy().view(np.uint64)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, (bad[:5], got[bad[:5]], want[bad[:5]])


def test_noalloc_reports_words_far_from_normalised(lnt):
    """Words whose carries do not settle within a block (here 2^40 over eight
    1-bit digits) return LNT_ERR_NUMERIC with the reason, not wrong digits."""
    import torch

    dev = torch.device("cuda", 0)
    fn = _noalloc()
    words = torch.full((8,), 1 << 40, dtype=torch.int64, device=dev)
    widths = torch.ones(8, dtype=torch.uint8, device=dev)
    out = torch.empty(8, dtype=torch.int64, device=dev)
    status = fn(words.data_ptr(), widths.data_ptr(), 8, 0, 0, out.data_ptr(),
                torch.cuda.current_stream(dev).cuda_stream)
    assert status == 5, status  # LNT_ERR_NUMERIC
    assert b"too far from normalised" in lnt.lib().lnt_last_error()
