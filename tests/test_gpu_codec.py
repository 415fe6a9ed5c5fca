"""A seed-compressed query end to end: the client builds its query around
c1 = Expand(seed) (the oracle client with that polynomial given), the codec
encodes it to 14,884 bytes and decodes it back, and the GPU answers the
decoded query bit for bit like the oracle server and decryptably."""
import numpy as np
import pytest

from onionpirv2_b200 import PirParams, PirServer
from onionpirv2_b200 import codec
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_decoded_query_is_answered_like_the_original():
    target, h, seed_db = 16384, 9, 11
    gp = PirParams(target, h)
    op = O.params(target, h)
    cl = O.Client(op, 77)
    seed = bytes((7 * i + 3) % 256 for i in range(32))
    a = codec.prf_expand(gp, seed, codec.PRF_QUERY, 0)
    idx = 4321
    q = cl.query_with_a(idx, a)
    assert np.array_equal(q[1], a)
    data = codec.encode_query(gp, seed, q)
    assert len(data) == 14884
    q2 = codec.decode_query(gp, data)
    assert np.array_equal(q2, q)
    srv = PirServer(gp)
    srv.load_data_seeded(target, seed_db)
    srv.set_client_keys(5, cl.bv_keys(), cl.gsw_key())
    resp = srv.make_query(5, q2)
    ref = O.Server(op)
    ref.load_seeded(target, seed_db)
    ref.set_keys(cl.bv_keys(), cl.gsw_key())
    assert np.array_equal(resp, ref.make_query(q))
    assert np.array_equal(cl.decrypt(resp), O.db_plaintext(seed_db, idx, op).astype(np.uint64))
