"""Session keys handed over in coefficient form (opir_server_set_client_keys_ex
with OPIR_KEYS_COEFF): the form a producer with another NTT convention -- a
client built on Intel HEXL -- obtains with its own inverse NTT. The server
takes every row into its NTT domain on the GPU; its answers must equal, bit
for bit, the answers with the same keys handed over in NTT form."""
import numpy as np
import pytest

from onionpirv2_b200 import PirParams, PirServer
from oracle import oracle as O

pytestmark = pytest.mark.gpu

C4 = "CONFIG_N4096_K2_MP"


def _intt_rows(keys: np.ndarray, mods, roots) -> np.ndarray:
    out = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    N = out.shape[-1]
    flat = out.reshape(-1, len(mods), N)
    for row in flat:
        for k, (q, w) in enumerate(zip(mods, roots)):
            poly = np.ascontiguousarray(row[k])
            O.lib().oracle_ntt_inv(O.ptr(poly), N, q, w)
            row[k] = poly
    return out


@pytest.mark.parametrize("config", ["k1", "c4"])
def test_coefficient_form_keys_answer_like_ntt_form(config):
    target, h, idx = 16384, 9, 777
    if config == "k1":
        gp, op = PirParams(target, h), O.params(target, h)
        cl = O.Client(op, 8)
        mods, roots = [int(op.q)], [int(op.w_crt)]
    else:
        gp, op = PirParams(target, h, config=C4), O.c4_params(target, h)
        cl = O.C4Client(op, 8)
        mods, roots = [int(x) for x in op.q[:2]], [int(x) for x in op.w[:2]]
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    bv_c, gsw_c = _intt_rows(bv, mods, roots), _intt_rows(gsw, mods, roots)
    assert not np.array_equal(bv_c, bv)
    srv = PirServer(gp)
    srv.load_data_seeded(target, 4)
    srv.set_client_keys(1, bv, gsw)
    srv.set_client_keys(2, bv_c, gsw_c, key_form="coeff")
    q = cl.query(idx)
    r1, r2 = srv.make_query(1, q), srv.make_query(2, q)
    assert np.array_equal(r1, r2)
    want = (O.db_plaintext(4, idx, op).astype(np.uint64) if config == "k1"
            else O.c4_db_plaintext(4, idx, op))
    assert np.array_equal(cl.decrypt(r2), want)
    bad = gsw_c.copy()
    bad.reshape(-1)[5] = mods[0]
    with pytest.raises(ValueError):
        srv.set_client_keys(3, bv_c, bad, key_form="coeff")
