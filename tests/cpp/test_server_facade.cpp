// Parity test of the C++ facade (include/onionpir_b200.hpp), written the way
// the reference's src/tests/test_pir.cpp and test_shared_session.cpp are: a
// server on a seeded database answers the queries of seeded clients that
// registered their keys (legacy setters or a shared session bundle); every
// response must equal the oracle server's bit for bit, serialize to the same
// bytes and decrypt to the plaintext recorded at load time. The public stage
// methods (expand_query, complete_selectors, evaluate_first_dim,
// evaluate_other_dim, ext_prod_mux) are checked against the oracle's stages,
// and the error paths against the reference's exception types. The client
// and the reference arithmetic come from the oracle (oracle/opir_oracle.h),
// the checker. Needs a GPU; prints "ok" and exits 0 on success.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "onionpir_b200.hpp"
#include "opir_oracle.h"

using namespace onionpir_b200;

namespace {

int failures = 0;

void require_test(bool ok, const std::string &what) {
  if (!ok) {
    std::fprintf(stderr, "FAIL: %s\n", what.c_str());
    ++failures;
  }
}

template <class E, class F>
void require_throws(F &&f, const std::string &what) {
  try {
    f();
  } catch (const E &) {
    return;
  } catch (const std::exception &e) {
    require_test(false, what + ": wrong exception (" + e.what() + ")");
    return;
  }
  require_test(false, what + ": no exception");
}

RlweCt to_ct(const uint64_t *flat, size_t kn) {
  RlweCt ct;
  ct.c0.assign(flat, flat + kn);
  ct.c1.assign(flat + kn, flat + 2 * kn);
  return ct;
}

std::vector<uint64_t> flat(const RlweCt &ct) {
  std::vector<uint64_t> f(ct.c0);
  f.insert(f.end(), ct.c1.begin(), ct.c1.end());
  return f;
}

// BV keys [level][row][b (kn)][a (kn)] and RGSW rows [row][c0 (kn)][c1 (kn)]
// as the reference's key objects.
bvks::BvGaloisKeys bv_keys_of(const std::vector<uint64_t> &bv, size_t h, size_t l_ks, size_t N,
                              size_t kn) {
  bvks::BvGaloisKeys keys;
  for (size_t d = 0; d < h; ++d) {
    bvks::BvKeySwitchKey k;
    k.galois_k = static_cast<uint32_t>(N / (1ull << d) + 1);
    for (size_t j = 0; j < l_ks; ++j) {
      const uint64_t *row = bv.data() + (d * l_ks + j) * 2 * kn;
      bvks::BvRlweCt ct;
      ct.b.assign(row, row + kn);
      ct.a.assign(row + kn, row + 2 * kn);
      k.cts.push_back(ct);
    }
    keys.keys.push_back(k);
  }
  return keys;
}

GSWCt gsw_of(const std::vector<uint64_t> &g, size_t rows, size_t kn) {
  GSWCt out;
  for (size_t r = 0; r < rows; ++r) out.emplace_back(g.data() + r * 2 * kn, g.data() + (r + 1) * 2 * kn);
  return out;
}

// ------------------------------------- CONFIG_N2048_K1_COMP and CONFIG_N2048_K1
// The one-limb sets: the oracle's routines take either set's parameters
// (init picks the set; CONFIG_N2048_K1 has one 60-bit prime).
void test_pir_one_limb(opir_config config,
                       int (*init)(uint64_t, uint32_t, int, opir_oracle_params *),
                       const std::string &label) {
  const uint64_t seed_db = 11;
  const size_t target = 16384, height = 9;
  PirParams pir_params = PirParams(config).with_layout({target, height, true});
  opir_oracle_params op;
  init(target, height, 1, &op);
  const size_t N = pir_params.get_poly_degree(), kn = pir_params.get_coeff_val_cnt();
  const size_t h = pir_params.get_expan_height(), l_ks = op.l_ks;
  require_test(pir_params.get_num_pt() == op.num_pt && pir_params.get_fst_dim_sz() == op.fst_dim_sz,
               label + " layout");

  PirServer server(pir_params);
  std::vector<size_t> query_indices = {0, 12345, target - 1};
  server.load_data(target, [&](size_t idx, RlwePt &pt) {
    std::vector<uint16_t> c(N);
    oracle_db_plaintext(seed_db, idx, &op, c.data());
    pt.data.assign(c.begin(), c.end());
  }, query_indices);
  oracle_server *ref = oracle_server_new(&op);
  oracle_server_load_seeded(ref, target, seed_db);

  oracle_client *last = nullptr;
  std::vector<uint64_t> last_query;
  for (size_t i = 0; i < query_indices.size(); ++i) {
    oracle_client *client = oracle_client_new(&op, 22 + i);
    const size_t client_id = 100 + i;
    std::vector<uint64_t> bv(h * l_ks * 2 * kn), g(2 * op.l_key * 2 * kn);
    oracle_client_bv_keys(client, bv.data());
    oracle_client_gsw_key(client, g.data());
    if (i == 1) {  // the multi-layout API: one shared immutable bundle
      auto bundle = std::make_shared<const PirSessionKeys>(
          PirSessionKeys{bv_keys_of(bv, h, l_ks, N, kn), gsw_of(g, 2 * op.l_key, kn)});
      server.set_client_session_keys(client_id, bundle);
      require_test(server.client_session_keys(client_id) == bundle, "session bundle kept");
    } else {
      server.set_client_bv_galois_key(client_id, bv_keys_of(bv, h, l_ks, N, kn));
      server.set_client_gsw_key(client_id, gsw_of(g, 2 * op.l_key, kn));
    }
    oracle_server_set_keys(ref, bv.data(), g.data());

    const size_t query_pt_idx = query_indices[i];
    std::vector<uint64_t> q(2 * kn);
    oracle_client_query(client, query_pt_idx, q.data());
    RlweCt query = to_ct(q.data(), kn);
    RlweCt response = server.make_query(client_id, query);

    std::vector<uint64_t> want(2 * N);
    oracle_server_make_query(ref, q.data(), want.data());
    require_test(flat(response) == want, label + " response bit-exact, index " + std::to_string(query_pt_idx));

    std::stringstream resp_stream;
    const size_t resp_size = server.save_resp_to_stream(response, resp_stream);
    std::vector<uint8_t> want_bytes(2 * N * 8);
    const size_t want_size = oracle_serialize(&op, want.data(), want_bytes.data());
    const std::string s = resp_stream.str();
    const std::vector<uint8_t> got_bytes(s.begin(), s.end());
    want_bytes.resize(want_size);
    require_test(resp_size == 11264 && resp_size == want_size && got_bytes == want_bytes,
                 label + " serialized response");

    std::vector<uint64_t> decrypted(N);
    std::vector<uint64_t> r = flat(response);
    oracle_client_decrypt(client, r.data(), decrypted.data());
    RlwePt actual_plaintext = server.direct_get_original_plaintext(query_pt_idx);
    require_test(decrypted == actual_plaintext.data, label + " decrypts to the recorded plaintext");
    if (last) oracle_client_free(last);
    last = client;
    last_query = q;
  }

  // the public stages (the tree-PIR callers' entry points) against the oracle
  const size_t client_id = 100 + query_indices.size() - 1;
  RlweCt query = to_ct(last_query.data(), kn);
  std::vector<RlweCt> expanded = server.expand_query(client_id, query);
  const size_t useful = op.fst_dim_sz + op.l_ep * (op.num_dims - 1);
  std::vector<uint64_t> e_want(useful * 2 * kn);
  oracle_server_expand(ref, last_query.data(), e_want.data());
  std::vector<uint64_t> e_got;
  for (const auto &ct : expanded) {
    const auto f = flat(ct);
    e_got.insert(e_got.end(), f.begin(), f.end());
  }
  require_test(expanded.size() == useful && e_got == e_want, label + " expand_query");

  std::vector<GSWCt> selectors = server.complete_selectors(client_id, expanded);
  std::vector<uint64_t> s_want((op.num_dims - 1) * 2 * op.l_ep * 2 * kn);
  oracle_server_complete_selectors(ref, e_want.data(), s_want.data());
  std::vector<uint64_t> s_got;
  for (const auto &gct : selectors)
    for (const auto &row : gct) s_got.insert(s_got.end(), row.begin(), row.end());
  require_test(s_got == s_want, label + " complete_selectors");

  std::vector<RlweCt> mid = server.evaluate_first_dim(expanded);
  std::vector<uint64_t> m_want(op.other_dim_sz * 2 * kn);
  oracle_server_first_dim(ref, e_want.data(), m_want.data());
  std::vector<uint64_t> m_got;
  for (const auto &ct : mid) {
    const auto f = flat(ct);
    m_got.insert(m_got.end(), f.begin(), f.end());
  }
  require_test(m_got == m_want, label + " evaluate_first_dim");

  RlweCt mux;
  server.ext_prod_mux(mid[0], mid[1], selectors[0], mux);
  std::vector<uint64_t> x(m_want.begin(), m_want.begin() + 2 * kn),
      y(m_want.begin() + 2 * kn, m_want.begin() + 4 * kn), mux_want(2 * kn);
  oracle_ext_prod_mux(&op, x.data(), y.data(), s_want.data(), mux_want.data());
  require_test(flat(mux) == mux_want, label + " ext_prod_mux");

  RlweCt fin = server.evaluate_other_dim(mid, selectors);
  std::vector<uint64_t> f_want(2 * kn);
  oracle_server_other_dim(ref, m_want.data(), s_want.data(), f_want.data());
  require_test(flat(fin) == f_want, label + " evaluate_other_dim");

  // error behaviour of the reference
  require_throws<std::out_of_range>([&] { server.make_query(999, query); }, "unknown client");
  RlweCt bad = query;
  bad.c0[0] = op.q;
  require_throws<std::invalid_argument>([&] { server.make_query(client_id, bad); },
                                        "unreduced query coefficient");
  require_throws<std::invalid_argument>([&] { server.direct_get_original_plaintext(5); },
                                        "unrecorded plaintext");
  require_throws<std::invalid_argument>(
      [&] { server.set_client_session_keys(7, nullptr); }, "null session bundle");
  require_throws<std::invalid_argument>(
      [&] { server.load_data(target, PlaintextSource{}); }, "missing source");
  require_throws<std::invalid_argument>(
      [&] { server.load_data(target + 1, [](size_t, RlwePt &) {}); }, "logical count beyond layout");
  require_throws<std::invalid_argument>(
      [&] {
        PirServer s2(pir_params);
        s2.load_data(4, [&](size_t, RlwePt &pt) { pt.data.assign(N, op.t); });
      },
      "coefficient above the plaintext modulus");
  require_throws<std::invalid_argument>(
      [&] {
        PirServer s2(pir_params);
        s2.load_data(4, [&](size_t, RlwePt &pt) { pt.data.assign(N - 1, 0); });
      },
      "wrong coefficient count");
  require_throws<std::invalid_argument>(
      [&] {
        PirServer qs(pir_params.with_query_shape({8, 2, 7}));
        qs.make_query(client_id, query);
      },
      "make_query on a query-shape view");
  require_throws<std::invalid_argument>([&] { PirParams().with_layout({16384, 40, true}); },
                                        "expansion height beyond log2 N");
  oracle_client_free(last);
  oracle_server_free(ref);
}

// ------------------------------- CONFIG_N4096_K2_MP and CONFIG_N2048_K2_MP
// The two-limb sets: the oracle's two-limb routines take either set's
// parameters (init picks the set).
void test_pir_two_limb(opir_config config,
                       int (*init)(uint64_t, uint32_t, int, opir_oracle_c4_params *),
                       size_t target, size_t height, size_t idx, size_t resp_bytes,
                       const std::string &label) {
  const uint64_t seed_db = 5;
  PirParams pir_params = PirParams(config).with_layout({target, height, true});
  opir_oracle_c4_params op;
  init(target, static_cast<uint32_t>(height), 1, &op);
  const size_t N = pir_params.get_poly_degree(), kn = pir_params.get_coeff_val_cnt();
  require_test(pir_params.K() == 2 && kn == 2 * N && N == op.N &&
                   pir_params.get_num_pt() == op.num_pt,
               label + " layout");
  PirServer server(pir_params);
  server.load_data(target, [&](size_t i, RlwePt &pt) {
    pt.data.resize(N);
    oracle_c4_db_plaintext(seed_db, i, &op, pt.data.data());
  }, {idx});
  oracle_c4_server *ref = oracle_c4_server_new(&op);
  oracle_c4_server_load_seeded(ref, target, seed_db);
  oracle_c4_client *client = oracle_c4_client_new(&op, 9);
  const size_t h = pir_params.get_expan_height();
  std::vector<uint64_t> bv(h * op.l_ks * 2 * kn), g(2 * op.l_key * 2 * kn);
  oracle_c4_client_bv_keys(client, bv.data());
  oracle_c4_client_gsw_key(client, g.data());
  server.set_client_bv_galois_key(3, bv_keys_of(bv, h, op.l_ks, N, kn));
  server.set_client_gsw_key(3, gsw_of(g, 2 * op.l_key, kn));
  oracle_c4_server_set_keys(ref, bv.data(), g.data());

  std::vector<uint64_t> q(2 * kn);
  oracle_c4_client_query(client, idx, q.data());
  RlweCt query = to_ct(q.data(), kn);
  RlweCt response = server.make_query(3, query);
  std::vector<uint64_t> want(2 * N);
  oracle_c4_server_make_query(ref, q.data(), want.data());
  require_test(flat(response) == want, label + " response bit-exact");
  std::stringstream resp_stream;
  require_test(server.save_resp_to_stream(response, resp_stream) == resp_bytes,
               label + " response bytes");
  std::vector<uint64_t> decrypted(N), r = flat(response);
  oracle_c4_client_decrypt(client, r.data(), decrypted.data());
  require_test(decrypted == server.direct_get_original_plaintext(idx).data,
               label + " decrypts to the recorded plaintext");

  // batched form (no counterpart in the reference) equals the single calls
  std::vector<RlweCt> qs = {query, query};
  std::vector<RlweCt> batch = server.make_query_batch({3, 3}, qs);
  require_test(batch.size() == 2 && flat(batch[0]) == want && flat(batch[1]) == want,
               label + " batch equals make_query");
  oracle_c4_client_free(client);
  oracle_c4_server_free(ref);
}

}  // namespace

int main() {
  test_pir_one_limb(OPIR_CONFIG_N2048_K1_COMP, oracle_params_init, "CONFIG_N2048_K1_COMP");
  test_pir_one_limb(OPIR_CONFIG_N2048_K1, oracle_k1p_params_init, "CONFIG_N2048_K1");
  test_pir_two_limb(OPIR_CONFIG_N4096_K2_MP, oracle_c4_params_init, 2048, 7, 777, 51200,
                    "CONFIG_N4096_K2_MP");
  test_pir_two_limb(OPIR_CONFIG_N2048_K2_MP, oracle_k2mp_params_init, 1000, 7, 777, 11264,
                    "CONFIG_N2048_K2_MP");
  if (failures) {
    std::fprintf(stderr, "%d check(s) failed\n", failures);
    return 1;
  }
  std::puts("ok");
  return 0;
}
