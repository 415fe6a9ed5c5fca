// Parity test of the C++ client facade GpuPirClient (include/onionpir_b200.hpp),
// written like the reference's src/tests/test_pir.cpp: a seeded client's
// secret, query randomness and key-generation randomness (from the oracle
// client, oracle/opir_oracle.h, the checker) go into the GPU client. Its
// session keys and queries must equal the oracle client's bit for bit, its
// decryptions the oracle's, and a server holding the GPU-made keys must answer
// GPU-made queries with responses that decrypt to the database plaintexts.
// Error paths are checked against the reference's exception types. Needs a
// GPU; prints "ok" and exits 0 on success.
#include <cstdio>
#include <memory>
#include <random>
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

std::vector<uint64_t> flat(const RlweCt &ct) {
  std::vector<uint64_t> f(ct.c0);
  f.insert(f.end(), ct.c1.begin(), ct.c1.end());
  return f;
}

// The GPU keys against the oracle's rows: BV [level][row][b][a], RGSW
// [row][c0][c1], each polynomial K*N values.
void compare_keys(const PirSessionKeys &keys, const std::vector<uint64_t> &bv,
                  const std::vector<uint64_t> &g, size_t h, size_t l_ks, size_t kn,
                  const std::string &tag) {
  bool ok = keys.bv_galois_keys.keys.size() == h;
  for (size_t d = 0; ok && d < h; ++d) {
    const auto &key = keys.bv_galois_keys.keys[d];
    for (size_t r = 0; r < l_ks; ++r) {
      const uint64_t *row = bv.data() + (d * l_ks + r) * 2 * kn;
      ok = ok && key.cts[r].b == std::vector<uint64_t>(row, row + kn) &&
           key.cts[r].a == std::vector<uint64_t>(row + kn, row + 2 * kn);
    }
  }
  require_test(ok, tag + " BV keys bit-exact");
  bool gok = true;
  for (size_t r = 0; r < keys.gsw_key.size(); ++r)
    gok = gok && keys.gsw_key[r] == std::vector<uint64_t>(g.begin() + r * 2 * kn,
                                                          g.begin() + (r + 1) * 2 * kn);
  require_test(gok && keys.gsw_key.size() * 2 * kn == g.size(), tag + " RGSW key bit-exact");
}

// ---------------------------------------------------------- CONFIG_N2048_K1_COMP
void test_client_k1() {
  const size_t target = 16384, height = 9, n = 40;  // n >= 32: the tensor-core forms
  const uint64_t seed_db = 5;
  PirParams pir_params = PirParams().with_layout({target, height, true});
  opir_oracle_params op;
  oracle_params_init(target, height, 1, &op);
  const size_t N = pir_params.get_poly_degree(), kn = pir_params.get_coeff_val_cnt();
  const size_t h = op.expansion_height, l_ks = op.l_ks, l_key = op.l_key;
  std::vector<uint64_t> bv_a(h * l_ks * kn), gsw_a(2 * l_key * kn);
  std::vector<int64_t> bv_e(h * l_ks * N), gsw_e(2 * l_key * N);
  oracle_client *cl = oracle_client_new_keygen_parts(&op, 31, bv_a.data(), bv_e.data(),
                                                     gsw_a.data(), gsw_e.data());
  std::vector<int8_t> s(N);
  oracle_client_secret(cl, s.data());
  GpuPirClient client(pir_params, s);

  const PirSessionKeys keys = client.create_session_keys(bv_a, bv_e, gsw_a, gsw_e);
  std::vector<uint64_t> bv(h * l_ks * 2 * kn), g(2 * l_key * 2 * kn);
  oracle_client_bv_keys(cl, bv.data());
  oracle_client_gsw_key(cl, g.data());
  compare_keys(keys, bv, g, h, l_ks, kn, "k1");

  std::mt19937_64 rng(77);
  std::vector<size_t> idx;
  std::vector<uint64_t> a(n * kn), want(n * 2 * kn);
  std::vector<int64_t> e(n * N);
  for (size_t i = 0; i < n; ++i) {
    idx.push_back(i == 0 ? 0 : i == 1 ? target - 1 : rng() % target);
    for (size_t j = 0; j < kn; ++j) a[i * kn + j] = rng() % op.q;
    oracle_client_query_parts(cl, idx[i], a.data() + i * kn, want.data() + i * 2 * kn,
                              e.data() + i * N);
  }
  std::vector<RlweCt> queries = client.fast_generate_queries(idx, a, e);
  bool qok = queries.size() == n;
  for (size_t i = 0; qok && i < n; ++i)
    qok = flat(queries[i]) == std::vector<uint64_t>(want.begin() + i * 2 * kn,
                                                     want.begin() + (i + 1) * 2 * kn);
  require_test(qok, "k1 queries bit-exact");
  const RlweCt one = client.fast_generate_query(idx[2], std::vector<uint64_t>(a.begin() + 2 * kn, a.begin() + 3 * kn),
                                                std::vector<int64_t>(e.begin() + 2 * N, e.begin() + 3 * N));
  require_test(flat(one) == flat(queries[2]), "k1 single query equals the batch's");

  PirServer server(pir_params);
  server.load_data(target, [&](size_t i, RlwePt &pt) {
    std::vector<uint16_t> c(N);
    oracle_db_plaintext(seed_db, i, &op, c.data());
    pt.data.assign(c.begin(), c.end());
  });
  server.set_client_session_keys(3, std::make_shared<const PirSessionKeys>(keys));
  std::vector<RlweCt> responses = server.make_query_batch(std::vector<size_t>(n, 3), queries);
  std::vector<uint64_t> noise;
  const std::vector<RlwePt> pts = client.decrypt_mod_q_batch(responses, &noise);
  bool dok = pts.size() == n && noise.size() == n;
  for (size_t i = 0; dok && i < n; ++i) {
    std::vector<uint16_t> c(N);
    oracle_db_plaintext(seed_db, idx[i], &op, c.data());
    std::vector<uint64_t> ref(N);
    oracle_client_decrypt(cl, flat(responses[i]).data(), ref.data());
    dok = pts[i].data == std::vector<uint64_t>(c.begin(), c.end()) && pts[i].data == ref &&
          noise[i] < op.small_q / (2 * op.t);
  }
  require_test(dok, "k1 responses decrypt to the database plaintexts");
  require_test(client.decrypt_mod_q(responses[0]).data == pts[0].data, "k1 single decryption");

  require_throws<std::out_of_range>(
      [&] { client.fast_generate_query(op.num_pt, std::vector<uint64_t>(kn), std::vector<int64_t>(N)); },
      "k1 index beyond the layout");
  require_throws<std::invalid_argument>(
      [&] { GpuPirClient bad(pir_params, std::vector<int8_t>(N, 2)); }, "k1 non-ternary secret");
  oracle_client_free(cl);
}

// ---------------------------------------------------------- CONFIG_N4096_K2_MP
void test_client_c4() {
  const size_t target = 16384, height = 9, n = 40;  // the tensor-core forms
  const uint64_t seed_db = 6;
  PirParams pir_params = PirParams(OPIR_CONFIG_N4096_K2_MP).with_layout({target, height, true});
  opir_oracle_c4_params op;
  oracle_c4_params_init(target, height, 1, &op);
  const size_t N = pir_params.get_poly_degree(), kn = pir_params.get_coeff_val_cnt();
  const size_t h = op.expansion_height, l_ks = op.l_ks, l_key = op.l_key;
  std::vector<uint64_t> bv_a(h * l_ks * kn), gsw_a(2 * l_key * kn);
  std::vector<int64_t> bv_e(h * l_ks * N), gsw_e(2 * l_key * N);
  oracle_c4_client *cl = oracle_c4_client_new_keygen_parts(&op, 32, bv_a.data(), bv_e.data(),
                                                           gsw_a.data(), gsw_e.data());
  std::vector<int8_t> s(N);
  oracle_c4_client_secret(cl, s.data());
  GpuPirClient client(pir_params, s);

  const PirSessionKeys keys = client.create_session_keys(bv_a, bv_e, gsw_a, gsw_e);
  std::vector<uint64_t> bv(h * l_ks * 2 * kn), g(2 * l_key * 2 * kn);
  oracle_c4_client_bv_keys(cl, bv.data());
  oracle_c4_client_gsw_key(cl, g.data());
  compare_keys(keys, bv, g, h, l_ks, kn, "c4");

  std::mt19937_64 rng(78);
  std::vector<size_t> idx;
  std::vector<uint64_t> a(n * kn), want(n * 2 * kn);
  std::vector<int64_t> e(n * N);
  for (size_t i = 0; i < n; ++i) {
    idx.push_back(rng() % target);
    for (size_t k = 0; k < 2; ++k)
      for (size_t j = 0; j < N; ++j) a[i * kn + k * N + j] = rng() % op.q[k];
    oracle_c4_client_query_parts(cl, idx[i], a.data() + i * kn, want.data() + i * 2 * kn,
                                 e.data() + i * N);
  }
  std::vector<RlweCt> queries = client.fast_generate_queries(idx, a, e);
  bool qok = true;
  for (size_t i = 0; i < n; ++i)
    qok = qok && flat(queries[i]) == std::vector<uint64_t>(want.begin() + i * 2 * kn,
                                                            want.begin() + (i + 1) * 2 * kn);
  require_test(qok, "c4 queries bit-exact");

  PirServer server(pir_params);
  server.load_data(target, [&](size_t i, RlwePt &pt) {
    pt.data.resize(N);
    oracle_c4_db_plaintext(seed_db, i, &op, pt.data.data());
  });
  server.set_client_bv_galois_key(4, keys.bv_galois_keys);
  server.set_client_gsw_key(4, keys.gsw_key);
  std::vector<RlweCt> responses = server.make_query_batch(std::vector<size_t>(n, 4), queries);
  const std::vector<RlwePt> pts = client.decrypt_mod_q_batch(responses);
  bool dok = true;
  for (size_t i = 0; i < n; ++i) {
    std::vector<uint64_t> plain(N), ref(N);
    oracle_c4_db_plaintext(seed_db, idx[i], &op, plain.data());
    oracle_c4_client_decrypt(cl, flat(responses[i]).data(), ref.data());
    dok = dok && pts[i].data == plain && pts[i].data == ref;
  }
  require_test(dok, "c4 responses decrypt to the database plaintexts");
  oracle_c4_client_free(cl);
}

}  // namespace

int main() {
  test_client_k1();
  test_client_c4();
  if (failures) {
    std::fprintf(stderr, "%d failure(s)\n", failures);
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
