// Seeded driver over the OnionPIRv2 reference's public API. Test
// infrastructure: it is linked with the unmodified reference sources (and the
// HEXL stand-in in oracle/hexl_standin) into oracle/_ref/opir_ref, and is used
//   (1) to generate the golden responses under tests/golden/ (mode "golden"),
//   (2) as the timed CPU baseline of PirServer::make_query (mode "time").
//
// The reference's own client seeds itself from std::random_device
// (client.cpp:20-23, bv_keyswitch.cpp:267, server.cpp:55). This driver keeps
// every algorithm of the reference and only supplies seeded generators:
//   * database: PirServer::load_data (server.cpp:80-203) with a seeded
//     counter-based PlaintextSource, coefficient = mix64(seed, pt*N+c) % t;
//   * secret key: gen_secret_key_rns (rlwe.cpp:219-228) on rng(client_seed);
//   * BV keys: bvks::gen_bv_ks_key (bv_keyswitch.cpp:222-259) for
//     galois_k = (N >> i) + 1, i < h (bv_keyswitch.cpp:270-274) on
//     rng(client_seed ^ kBvSalt) -- the reference draws these from a
//     generator separate from the client's own;
//   * RGSW(s): GSWEval::plain_to_gsw (gsw.cpp:359-422) as in
//     PirClient::generate_gsw_from_key (client.cpp:25-38) on rng(client_seed);
//   * query: PirClient::fast_generate_query / add_gsw_to_query
//     (client.cpp:48-225) restated over the same public helpers on
//     rng(client_seed), continuing after the RGSW key draws;
//   * tree query (mode "tree"): make_tree_query (tree_query.cpp:142-196)
//     with PirClient::fresh_zero_ct's encryption of zero on the same
//     generator and the reference's own add_bfv_query_constant /
//     add_rlwe_star_constant; the server side (unpack_tree_query,
//     build_alpha_pyramid, preprocess_tree_reference, select_level) is the
//     reference's code unchanged.
#include "bv_keyswitch.h"
#include "client.h"
#include "gsw.h"
#include "pir.h"
#include "rlwe.h"
#include "server.h"
#include "tree_index.h"
#include "tree_query.h"
#include "tree_select.h"
#include "utils.h"
#include "hexl/hexl.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include <sys/wait.h>
#include <unistd.h>

namespace {

constexpr uint64_t kBvSalt = 0x5BD1E9955BD1E995ULL;
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

uint64_t db_coeff(uint64_t seed, uint64_t pt, uint64_t c, uint64_t n, uint64_t t) {
  return mix64(seed + (pt * n + c + 1) * kGolden) % t;
}

struct Client {
  RlweSk sk;
  bvks::BvGaloisKeys bv;
  GSWCt gsw;
  std::mt19937_64 rng;
};

Client make_client(const PirParams &p, uint64_t seed) {
  constexpr size_t N = DBConsts::PolyDegree;
  Client c{{}, {}, {}, std::mt19937_64(seed)};
  const std::vector<uint64_t> qs(p.get_rns_mods().begin(), p.get_rns_mods().end());
  c.sk = gen_secret_key_rns(N, qs, c.rng);
  std::mt19937_64 rng_bv(seed ^ kBvSalt);
  for (size_t i = 0; i < p.get_expan_height(); ++i) {
    const uint32_t galois_k = static_cast<uint32_t>((N >> i) + 1);
    c.bv.keys.push_back(bvks::gen_bv_ks_key(p, c.sk, galois_k, rng_bv));
  }
  std::vector<uint64_t> sk_coef(c.sk.data.begin(), c.sk.data.begin() + N);
  utils::ntt_inv(sk_coef.data(), N, qs[0]);
  GSWEval key_gsw(p, p.get_l_key(), p.get_base_log2_key());
  c.gsw = key_gsw.plain_to_gsw(sk_coef, c.sk, c.rng);
  return c;
}

// client.cpp:48-98
std::vector<size_t> query_indices(const PirParams &p, size_t pt_idx) {
  const size_t col = pt_idx % p.get_fst_dim_sz();
  const size_t row = pt_idx / p.get_fst_dim_sz();
  const size_t other = p.get_other_dim_sz();
  const size_t d = p.get_num_dims();
  std::vector<size_t> out = {col};
  if (d == 1) return out;
  const size_t h = d - 1;
  const size_t r = 2 * other - (size_t{1} << h);
  const size_t sl = other - r;
  size_t perfect;
  if (row < sl) {
    out.push_back(0);
    perfect = row;
  } else {
    const size_t corrected = row - sl;
    out.push_back(corrected % 2);
    perfect = sl + corrected / 2;
  }
  if (h > 1) {
    for (size_t k = h - 2; k + 1 > 0; k--) {
      out.push_back((perfect >> k) & 1ULL);
      if (k == 0) break;
    }
  }
  return out;
}

// client.cpp:107-225 (both branches: K = 1, the logical composite modulus;
// K = 2, two RNS limbs with the message lifted under Q = q0 q1).
RlweCt make_query(const PirParams &p, Client &c, size_t pt_idx) {
  constexpr size_t N = DBConsts::PolyDegree;
  const std::vector<uint64_t> qs(p.get_rns_mods().begin(), p.get_rns_mods().end());
  const size_t K = qs.size();
  const uint64_t t = p.get_plain_mod();
  const std::vector<size_t> qi = query_indices(p, pt_idx);
  const size_t h = p.get_expan_height();
  const size_t capacity = size_t{1} << h;
  uint64_t inverse = 0;
  utils::try_invert_uint_mod(capacity, t, inverse);
  const size_t rev = utils::bit_reverse(qi[0], h);
  RlweCt query;
  encrypt_zero_rns(c.sk, N, qs, p.get_noise_std_dev(), c.rng, query, false);
  if (K == 1) {
    const uint64_t Q = qs[0];
    const uint64_t scaled = utils::round_div_u128((uint128_t)Q * inverse, t) % Q;
    query.c0[rev] = (query.c0[rev] + scaled) % Q;
  } else {
    const uint128_t Q = (uint128_t)qs[0] * qs[1];
    const uint128_t Delta = Q / t;
    const uint64_t r = (uint64_t)(Q - Delta * t);
    const uint64_t r_inv_round = (uint64_t)(((uint128_t)r * inverse + (t >> 1)) / t);
    const uint128_t scaled_mp = Delta * inverse + r_inv_round;
    for (size_t k = 0; k < K; ++k) {
      const uint64_t sk = (uint64_t)(scaled_mp % qs[k]);
      query.c0[k * N + rev] = (uint64_t)(((uint128_t)query.c0[k * N + rev] + sk) % qs[k]);
    }
  }
  if (qi.size() > 1) {
    std::vector<uint64_t> inv_cap(K);
    for (size_t k = 0; k < K; ++k) utils::try_invert_uint_mod(capacity, qs[k], inv_cap[k]);
    const auto gadget = utils::gsw_gadget(p.get_l(), p.get_base_log2(), qs);
    for (size_t i = 1; i < qi.size(); i++) {
      if (qi[i] != 1) continue;
      for (size_t k = 0; k < p.get_l(); k++) {
        const size_t pos = p.get_fst_dim_sz() + (i - 1) * p.get_l() + k;
        const size_t ridx = utils::bit_reverse(pos, h);
        for (size_t m = 0; m < K; ++m) {
          const uint64_t coef = (uint64_t)((uint128_t)gadget[m][k] * inv_cap[m] % qs[m]);
          query.c0[m * N + ridx] = (uint64_t)(((uint128_t)query.c0[m * N + ridx] + coef) % qs[m]);
        }
      }
    }
  }
  return query;
}

// client.cpp:364-430, decryption under small_q.
RlwePt decrypt_small_q(const PirParams &p, const Client &c, const RlweCt &ct) {
  constexpr size_t N = DBConsts::PolyDegree;
  const uint64_t q = p.get_small_q();
  const uint64_t t = p.get_plain_mod();
  std::vector<uint64_t> sk_coef(c.sk.data.begin(), c.sk.data.begin() + N);
  utils::ntt_inv(sk_coef.data(), N, p.get_rns_mods()[0]);
  std::vector<uint64_t> sks(N), c0(N), c1(N), phase(N);
  for (size_t i = 0; i < N; i++) sks[i] = (sk_coef[i] > 1) ? (q - 1) : sk_coef[i];
  utils::ntt_fwd(sks.data(), N, q);
  for (size_t i = 0; i < N; i++) { c0[i] = ct.c0[i] % q; c1[i] = ct.c1[i] % q; }
  utils::ntt_fwd(c1.data(), N, q);
  intel::hexl::EltwiseMultMod(phase.data(), c1.data(), sks.data(), N, q, 1);
  utils::ntt_inv(phase.data(), N, q);
  intel::hexl::EltwiseAddMod(phase.data(), phase.data(), c0.data(), N, q);
  RlwePt out;
  out.data.resize(N);
  for (size_t i = 0; i < N; i++)
    out.data[i] = utils::round_div_u128((uint128_t)phase[i] * t, q) % t;
  return out;
}

void write_u64(const std::string &path, const std::vector<uint64_t> &v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char *>(v.data()), v.size() * 8);
}

struct Args {
  std::string mode = "golden";
  size_t target = 16384, height = 9;
  bool pow2 = true;
  uint64_t db_seed = 1, client_seed = 2;
  size_t index = 0;
  size_t queries = 1, warmup = 0, procs = 1;
  std::string out;
  bool dump_inputs = false;
  std::string stages;  // directory for the public stage outputs (golden mode)
  size_t tree_L = 16, tree_a = 3, leaf = 0;  // mode "tree"
};

Args parse(int argc, char **argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    std::string k = argv[i];
    auto val = [&]() -> std::string {
      if (i + 1 >= argc) throw std::invalid_argument("missing value for " + k);
      return argv[++i];
    };
    if (k == "--mode") a.mode = val();
    else if (k == "--target") a.target = std::stoull(val());
    else if (k == "--height") a.height = std::stoull(val());
    else if (k == "--pow2") a.pow2 = std::stoull(val()) != 0;
    else if (k == "--db-seed") a.db_seed = std::stoull(val());
    else if (k == "--client-seed") a.client_seed = std::stoull(val());
    else if (k == "--index") a.index = std::stoull(val());
    else if (k == "--queries") a.queries = std::stoull(val());
    else if (k == "--warmup") a.warmup = std::stoull(val());
    else if (k == "--procs") a.procs = std::stoull(val());
    else if (k == "--out") a.out = val();
    else if (k == "--dump-inputs") a.dump_inputs = true;
    else if (k == "--stages") a.stages = val();
    else if (k == "--tree-L") a.tree_L = std::stoull(val());
    else if (k == "--tree-a") a.tree_a = std::stoull(val());
    else if (k == "--leaf") a.leaf = std::stoull(val());
    else throw std::invalid_argument("unknown option " + k);
  }
  return a;
}

}  // namespace

// Mode "tree": one packed tree query for `leaf` through the reference's tree
// layer on the default scheme (as src/tests/test_tree_select.cpp does);
// writes query.u64, alpha.u64, beta.u64 (the beta selectors) and levels.u64
// (select_level of every level, c0 || c1 each) into --out and prints whether
// every level decrypts to its packed plaintext D_l[p_l].
int run_tree(const Args &a) {
  constexpr size_t N = DBConsts::PolyDegree;
  PirParams scheme;
  const TreePirParams tree = make_tree_pir_params_for_scheme(a.tree_L, a.tree_a, scheme);
  Client c = make_client(scheme, a.client_seed);
  const std::vector<uint64_t> qs(scheme.get_rns_mods().begin(), scheme.get_rns_mods().end());
  // make_tree_query (tree_query.cpp:142-196)
  const ClientCoordinates coords = client_index(a.leaf, tree);
  RlweCt query;
  encrypt_zero_rns(c.sk, N, qs, scheme.get_noise_std_dev(), c.rng, query, false);
  const uint64_t t = scheme.get_plain_mod();
  uint64_t w_inv_t = 0;
  utils::try_invert_uint_mod(tree.W, t, w_inv_t);
  add_bfv_query_constant(query, scheme, coords.alpha, tree.h_q, w_inv_t);
  const size_t K = qs.size();
  std::vector<uint64_t> w_inv_q(K);
  for (size_t k = 0; k < K; ++k) utils::try_invert_uint_mod(tree.W, qs[k], w_inv_q[k]);
  const size_t ell = scheme.get_l();
  const auto gadget = utils::gsw_gadget(ell, scheme.get_base_log2(), qs);
  std::vector<uint64_t> vals(K);
  auto rows = [&](size_t group) {
    for (size_t row = 0; row < ell; ++row) {
      for (size_t k = 0; k < K; ++k)
        vals[k] = (uint64_t)((uint128_t)gadget[k][row] * w_inv_q[k] % qs[k]);
      add_rlwe_star_constant(query, scheme, tree.N0 + group * ell + row, tree.h_q, vals);
    }
  };
  for (size_t u = 0; u < tree.b; ++u) if (coords.beta_bits_le[u]) rows(u);
  for (size_t v = 0; v < tree.r; ++v) if (coords.gamma_bits_le[v]) rows(tree.b + v);

  std::vector<uint64_t> v(query.c0);
  v.insert(v.end(), query.c1.begin(), query.c1.end());
  write_u64(a.out + "/query.u64", v);
  PirServer server(tree_query_expansion_params(tree, scheme));
  server.set_client_bv_galois_key(1, c.bv);
  server.set_client_gsw_key(1, c.gsw);
  const TreeNodeSource source = [&](size_t level, size_t index) {
    return synthetic_tree_node_value(level, index, t);
  };
  const std::vector<TreeLevelDatabase> levels = preprocess_tree_reference(tree, source);
  const std::vector<LevelPlan> plans = build_level_plans(tree);
  // server-side time of one tree query: unpack + every level's select_level
  const auto t0 = std::chrono::steady_clock::now();
  RlweCt qcopy = query;
  ExpandedTreeQuery un = unpack_tree_query(server, scheme, tree, 1, qcopy);
  const AlphaPyramid pyramid = build_alpha_pyramid(un.alpha, tree, scheme);
  std::vector<RlweCt> selected;
  for (size_t level = 0; level <= tree.L; ++level)
    selected.push_back(select_level(levels[level], plans[level], pyramid,
                                    std::span<GSWCt>(un.beta_selectors), server, tree, scheme));
  const double server_ms = std::chrono::duration<double, std::milli>(
      std::chrono::steady_clock::now() - t0).count();
  v.clear();
  for (const auto &ct : un.alpha) { v.insert(v.end(), ct.c0.begin(), ct.c0.end());
                                    v.insert(v.end(), ct.c1.begin(), ct.c1.end()); }
  write_u64(a.out + "/alpha.u64", v);
  v.clear();
  for (const auto &g : un.beta_selectors) for (const auto &row : g) v.insert(v.end(), row.begin(), row.end());
  write_u64(a.out + "/beta.u64", v);
  bool ok = true;
  v.clear();
  for (size_t level = 0; level <= tree.L; ++level) {
    const RlweCt &sel = selected[level];
    v.insert(v.end(), sel.c0.begin(), sel.c0.end());
    v.insert(v.end(), sel.c1.begin(), sel.c1.end());
    RlwePt dec;
    decrypt_rns(sel, c.sk, N, qs, t, scheme.get_rns_tables(), dec);
    const LevelOracle oracle = build_level_oracle_for_test(a.leaf, level, tree);
    ok = ok && dec.data == levels[level].plaintexts[oracle.packed_plaintext_index];
  }
  write_u64(a.out + "/levels.u64", v);
  std::printf("{\"ok\": %s, \"N0\": %zu, \"b\": %zu, \"r\": %zu, \"h_q\": %zu, \"w\": %zu, "
              "\"alpha\": %zu, \"server_ms\": %.3f}\n", ok ? "true" : "false", tree.N0, tree.b,
              tree.r, tree.h_q, tree.w, coords.alpha, server_ms);
  return ok ? 0 : 3;
}

int main(int argc, char **argv) {
  try {
    const Args a = parse(argc, argv);
    if (a.mode == "tree") return run_tree(a);
    constexpr size_t N = DBConsts::PolyDegree;
    PirParams params = PirParams().with_layout({a.target, a.height, a.pow2});
    const uint64_t t = params.get_plain_mod();
    PirServer server(params);
    const uint64_t seed = a.db_seed;
    PlaintextSource source = [&](size_t idx, RlwePt &out) {
      out.data.resize(N);
      for (size_t c = 0; c < N; ++c) out.data[c] = db_coeff(seed, idx, c, N, t);
    };
    const auto t_load0 = std::chrono::steady_clock::now();
    std::vector<size_t> record;
    if (a.mode == "golden") record.push_back(a.index);
    server.load_data(a.target, source, record);
    const double load_s = std::chrono::duration<double>(
        std::chrono::steady_clock::now() - t_load0).count();

    if (a.mode == "golden") {
      Client c = make_client(params, a.client_seed);
      server.set_client_bv_galois_key(1, c.bv);
      server.set_client_gsw_key(1, c.gsw);
      RlweCt query = make_query(params, c, a.index);
      RlweCt query_copy = query;
      if (!a.stages.empty()) {
        // PirServer's public stage methods (server.h:43-99) on a copy of the
        // query, each written as flat u64 in the reference's own layouts
        RlweCt q2 = query;
        std::vector<RlweCt> exp = server.expand_query(1, q2);
        std::vector<uint64_t> v;
        for (const auto &ct : exp) { v.insert(v.end(), ct.c0.begin(), ct.c0.end());
                                     v.insert(v.end(), ct.c1.begin(), ct.c1.end()); }
        write_u64(a.stages + "/expand.u64", v);
        std::vector<GSWCt> sel = server.complete_selectors(1, exp);
        v.clear();
        for (const auto &g : sel) for (const auto &row : g) v.insert(v.end(), row.begin(), row.end());
        write_u64(a.stages + "/selectors.u64", v);
        exp.resize(params.get_fst_dim_sz());
        std::vector<RlweCt> mid = server.evaluate_first_dim(exp);
        v.clear();
        for (const auto &ct : mid) { v.insert(v.end(), ct.c0.begin(), ct.c0.end());
                                     v.insert(v.end(), ct.c1.begin(), ct.c1.end()); }
        write_u64(a.stages + "/first_dim.u64", v);
        RlweCt fin = server.evaluate_other_dim(mid, sel);
        v.assign(fin.c0.begin(), fin.c0.end());
        v.insert(v.end(), fin.c1.begin(), fin.c1.end());
        write_u64(a.stages + "/other_dim.u64", v);
      }
      RlweCt resp = server.make_query(1, query);
      std::stringstream ss;
      const size_t nbytes = server.save_resp_to_stream(resp, ss);
      const std::string stream = ss.str();
      RlwePt dec = decrypt_small_q(params, c, resp);
      RlwePt want = server.direct_get_original_plaintext(a.index);
      const bool ok = dec.data == want.data;
      if (!a.out.empty()) {
        std::vector<uint64_t> r(resp.c0);
        r.insert(r.end(), resp.c1.begin(), resp.c1.end());
        write_u64(a.out + "/response.u64", r);
        std::ofstream(a.out + "/response.bin", std::ios::binary).write(stream.data(), stream.size());
        if (a.dump_inputs) {
          std::vector<uint64_t> qv(query_copy.c0);
          qv.insert(qv.end(), query_copy.c1.begin(), query_copy.c1.end());
          write_u64(a.out + "/query.u64", qv);
          std::vector<uint64_t> kv;
          for (const auto &key : c.bv.keys)
            for (const auto &row : key.cts) {
              kv.insert(kv.end(), row.b.begin(), row.b.end());
              kv.insert(kv.end(), row.a.begin(), row.a.end());
            }
          write_u64(a.out + "/bv_keys.u64", kv);
          std::vector<uint64_t> gv;
          for (const auto &row : c.gsw) gv.insert(gv.end(), row.begin(), row.end());
          write_u64(a.out + "/gsw_key.u64", gv);
        }
      }
      const auto &crt = params.get_composite_rns();
      const auto &qs = params.get_rns_mods();
      std::printf(
          "{\"ok\": %s, \"num_pt\": %zu, \"fst_dim_sz\": %zu, \"num_dims\": %zu, "
          "\"other_dim_sz\": %zu, \"K\": %zu, \"q\": %llu, \"q_limb1\": %llu, \"q1\": %llu, "
          "\"q2\": %llu, \"w1\": %llu, \"w2\": %llu, \"t\": %llu, \"small_q\": %llu, "
          "\"base_log2\": %zu, \"base_log2_key\": %zu, \"resp_bytes\": %zu, \"load_s\": %.3f}\n",
          ok ? "true" : "false", params.get_num_pt(), params.get_fst_dim_sz(),
          params.get_num_dims(), params.get_other_dim_sz(), qs.size(),
          (unsigned long long)qs[0], (unsigned long long)(qs.size() > 1 ? qs[1] : 0),
          (unsigned long long)crt.q1, (unsigned long long)crt.q2, (unsigned long long)crt.w1,
          (unsigned long long)crt.w2, (unsigned long long)t,
          (unsigned long long)params.get_small_q(), (size_t)params.get_base_log2(),
          (size_t)params.get_base_log2_key(), nbytes, load_s);
      return ok ? 0 : 3;
    }

    if (a.mode == "time") {
      // The timer boundary is make_query only (merkle_benchmark.cpp:549-553).
      // P processes are forked after load_data so the preprocessed database
      // is shared copy-on-write; each runs its own clients and queries.
      const int P = static_cast<int>(a.procs < 1 ? 1 : a.procs);
      std::vector<int> fds(P);
      std::vector<pid_t> pids(P);
      for (int p = 0; p < P; ++p) {
        int fd[2];
        if (pipe(fd) != 0) throw std::runtime_error("pipe");
        const pid_t pid = fork();
        if (pid < 0) throw std::runtime_error("fork");
        if (pid == 0) {
          close(fd[0]);
          double sum_ms = 0, wall_ms = 0;
          size_t failures = 0, timed = 0;
          std::chrono::steady_clock::time_point wall0;
          for (size_t q = 0; q < a.warmup + a.queries; ++q) {
            const uint64_t cseed = a.client_seed + 1000003ull * p + q;
            Client c = make_client(params, cseed);
            server.set_client_bv_galois_key(q + 1, c.bv);
            server.set_client_gsw_key(q + 1, c.gsw);
            const size_t idx = static_cast<size_t>(mix64(cseed * 7919) % a.target);
            RlweCt query = make_query(params, c, idx);
            if (q == a.warmup) wall0 = std::chrono::steady_clock::now();
            const auto t0 = std::chrono::steady_clock::now();
            RlweCt resp = server.make_query(q + 1, query);
            const double dt = std::chrono::duration<double, std::milli>(
                std::chrono::steady_clock::now() - t0).count();
            RlwePt dec = decrypt_small_q(params, c, resp);
            for (size_t i = 0; i < N; ++i)
              if (dec.data[i] != db_coeff(seed, idx, i, N, t)) { ++failures; break; }
            if (q >= a.warmup) { sum_ms += dt; ++timed; }
          }
          if (timed) wall_ms = std::chrono::duration<double, std::milli>(
              std::chrono::steady_clock::now() - wall0).count();
          char buf[256];
          const int n = std::snprintf(buf, sizeof buf, "%.6f %.6f %zu %zu\n", sum_ms, wall_ms,
                                      timed, failures);
          if (write(fd[1], buf, n) != n) _exit(2);
          close(fd[1]);
          _exit(0);
        }
        close(fd[1]);
        fds[p] = fd[0];
        pids[p] = pid;
      }
      double sum_ms = 0, wall_max = 0;
      size_t timed = 0, failures = 0;
      for (int p = 0; p < P; ++p) {
        char buf[256] = {0};
        const ssize_t n = read(fds[p], buf, sizeof buf - 1);
        close(fds[p]);
        int status = 0;
        waitpid(pids[p], &status, 0);
        double s1 = 0, w1 = 0;
        size_t t1 = 0, f1 = 0;
        if (n <= 0 || std::sscanf(buf, "%lf %lf %zu %zu", &s1, &w1, &t1, &f1) != 4 ||
            !WIFEXITED(status) || WEXITSTATUS(status) != 0)
          throw std::runtime_error("timing child failed");
        sum_ms += s1;
        timed += t1;
        failures += f1;
        wall_max = std::max(wall_max, w1);
      }
      const double mean = timed ? sum_ms / timed : 0.0;
      const double qps = wall_max > 0 ? timed / (wall_max / 1000.0) : 0.0;
      std::printf("{\"mean_ms\": %.3f, \"qps\": %.4f, \"queries\": %zu, \"procs\": %d, "
                  "\"failures\": %zu, \"load_s\": %.3f}\n",
                  mean, qps, timed, P, failures, load_s);
      return failures ? 3 : 0;
    }
    throw std::invalid_argument("unknown mode " + a.mode);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "opir_ref error: %s\n", e.what());
    return 1;
  }
}
