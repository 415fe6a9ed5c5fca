"""The allocation-free MUX entry point (opir_ext_prod_mux_noalloc).

It exists for callers that cannot allocate device memory when they run a MUX
step (a host that owns and pre-budgets all device memory, or a request loop
that must stay off the CUDA allocator). The test calls it through the C ABI
on buffers the test itself allocates, twice in a row and as a batch, and
checks every output bit for bit against the existing entry point
(opir_server_evaluate_other_dim on a one-MUX layout) and against the CPU
oracle's ext_prod_mux. This file is collected last so a failure here never
hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from onionpirv2_b200 import PirParams, PirServer
from onionpirv2_b200 import _lib as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _inputs(p, n, seed):
    rng = np.random.default_rng(seed)
    x = rng.integers(0, p.q, (n, 2, p.N), dtype=np.uint64)
    y = rng.integers(0, p.q, (n, 2, p.N), dtype=np.uint64)
    sel = rng.integers(0, p.q, (n, 2 * p.l_ep, 2, p.N), dtype=np.uint64)
    return x, y, sel


def _expected(p, x, y, sel):
    # layout 43 / h5 / non-pow2: two candidates and one selector, so
    # evaluate_other_dim is exactly one ext_prod_mux(x, y, sel)
    assert p.num_dims == 2 and p.other_dim_sz == 2
    with PirServer(p) as srv:
        return np.stack([srv.evaluate_other_dim(np.stack([x[i], y[i]]), sel[i][None])
                         for i in range(x.shape[0])])


def _noalloc(p, x, y, sel, side_stream=False):
    import torch
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).to(dev)
    dx, dy, ds = t(x), t(y), t(sel)
    dout = torch.empty_like(dx)
    lib = L.load()
    stream = torch.cuda.Stream(dev) if side_stream else None
    if stream is not None:
        stream.wait_stream(torch.cuda.current_stream(dev))   # the inputs are on the device
    rc = lib.opir_ext_prod_mux_noalloc(C.byref(p._p), x.shape[0], dx.data_ptr(), dy.data_ptr(),
                                       ds.data_ptr(), dout.data_ptr(),
                                       C.c_void_p(stream.cuda_stream) if stream else None)
    torch.cuda.synchronize(dev)
    assert rc == 0
    return dout.cpu().numpy().view(np.uint64)


def _oracle(p, x, y, sel):
    op = O.params(43, 5, False)
    assert (op.q, op.N, op.l_ep) == (p.q, p.N, p.l_ep)
    return np.stack([O.ext_prod_mux(op, x[i], y[i], sel[i]) for i in range(x.shape[0])])


def test_noalloc_mux_matches_existing_entry_point_twice():
    p = PirParams(43, 5, False)
    x, y, sel = _inputs(p, 1, 11)
    want = _expected(p, x, y, sel)
    first = _noalloc(p, x, y, sel)
    second = _noalloc(p, x, y, sel)
    assert np.array_equal(first, want)
    assert np.array_equal(second, want)
    assert np.array_equal(first, _oracle(p, x, y, sel))


def test_noalloc_mux_on_a_side_stream_and_parameter_check():
    p = PirParams(43, 5, False)
    x, y, sel = _inputs(p, 2, 14)
    want = _oracle(p, x, y, sel)
    assert np.array_equal(_noalloc(p, x, y, sel), want)
    assert np.array_equal(_noalloc(p, x, y, sel, side_stream=True), want)
    # the fixed tables hold one modulus: other moduli are refused
    bad = type(p._p).from_buffer_copy(p._p)
    bad.q = p.q - 2
    import torch
    buf = torch.zeros(2 * p.l_ep * 2 * p.N, dtype=torch.int64, device="cuda")
    rc = L.load().opir_ext_prod_mux_noalloc(C.byref(bad), 1, buf.data_ptr(), buf.data_ptr(),
                                            buf.data_ptr(), buf.data_ptr(), None)
    assert rc == 1   # OPIR_ERR_INVALID_ARGUMENT


def test_noalloc_mux_batch_and_limit():
    p = PirParams(43, 5, False)
    x, y, sel = _inputs(p, 3, 12)
    assert np.array_equal(_noalloc(p, x, y, sel), _expected(p, x, y, sel))
    # a different batch right after: results depend only on this call's inputs
    x2, y2, sel2 = _inputs(p, 2, 13)
    assert np.array_equal(_noalloc(p, x2, y2, sel2), _expected(p, x2, y2, sel2))
    # more MUX steps than the fixed working memory holds are refused
    import torch
    big = torch.zeros(9 * 2 * p.N, dtype=torch.int64, device="cuda")
    sbig = torch.zeros(9 * 2 * p.l_ep * 2 * p.N, dtype=torch.int64, device="cuda")
    rc = L.load().opir_ext_prod_mux_noalloc(C.byref(p._p), 9, big.data_ptr(), big.data_ptr(),
                                            sbig.data_ptr(), big.data_ptr(), None)
    assert rc == 1   # OPIR_ERR_INVALID_ARGUMENT
