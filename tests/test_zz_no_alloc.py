"""GPU: the allocation-free readout (lnt_canonicalize_noalloc) against lnt_get_digits.

Some callers cannot allocate device memory when they need a residue in the
reference's digit format: a serving process that has handed all of its HBM to
its own pool or admission budget, a latency-critical step that must not pay
cudaMalloc's implicit device synchronisation, a checkpoint written from an
interrupt handler.  They pass their own device buffers to
lnt_canonicalize_noalloc, whose scratch is one fixed library-owned array
(residues up to 2^24 words).  Its digits must equal the regular readout's
exactly (integer digits: the tolerance is zero), on two calls in a row that
share that array.

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
