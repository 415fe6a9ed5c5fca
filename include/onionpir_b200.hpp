// C++ facade of the reference's server interface over the C ABI of
// onionpir_b200.h: the class and method names, argument meaning, data
// layouts and exception types of PirServer / PirParams and their value types
// (includes/server.h:13-172, pir.h:35-167, rlwe.h:17-49, gsw.h:17,
// bv_keyswitch.h:48-66, pir_session.h:8-18), so code written
// against the reference's server reads the same against this library.
// Header-only C++17; link with libonionpir_b200.so. The value types live in
// namespace onionpir_b200 (they are layout-identical to the reference's, so a
// caller that also builds the reference client copies vectors across).
//
// Status codes become the exceptions the reference throws:
// OPIR_ERR_INVALID_ARGUMENT -> std::invalid_argument, OPIR_ERR_OUT_OF_RANGE
// -> std::out_of_range, OPIR_ERR_OVERFLOW -> std::overflow_error,
// OPIR_ERR_NO_MEMORY -> std::bad_alloc, anything else -> std::runtime_error.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <exception>
#include <functional>
#include <map>
#include <memory>
#include <new>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "onionpir_b200.h"

namespace onionpir_b200 {

// ------------------------------------------------------------- value types
// RlweCt (rlwe.h:17-31): c0, c1 of K*N values each, limb-major.
struct RlweCt {
  std::vector<uint64_t> c0;
  std::vector<uint64_t> c1;
  bool ntt_form = false;

  uint64_t *data(size_t i) { return i == 0 ? c0.data() : c1.data(); }
  const uint64_t *data(size_t i) const { return i == 0 ? c0.data() : c1.data(); }
  bool &is_ntt_form() { return ntt_form; }
  void resize(size_t n) { c0.assign(n, 0); c1.assign(n, 0); }
  size_t poly_size() const { return c0.size(); }
};

// RlwePt (rlwe.h:46-49): N coefficients in [0, t).
struct RlwePt {
  std::vector<uint64_t> data;
  size_t coeff_count() const { return data.size(); }
};

// GSWCt (gsw.h:17): 2 l rows, each [c0 (K*N)][c1 (K*N)], NTT form.
typedef std::vector<std::vector<uint64_t>> GSWCt;

namespace bvks {
// BvRlweCt / BvKeySwitchKey / BvGaloisKeys (bv_keyswitch.h:48-66): a = c1
// part, b = c0 part, K*N values each, NTT form.
struct BvRlweCt {
  std::vector<uint64_t> a;
  std::vector<uint64_t> b;
};
struct BvKeySwitchKey {
  uint32_t galois_k = 0;
  std::vector<BvRlweCt> cts;
};
class BvGaloisKeys {
 public:
  std::vector<BvKeySwitchKey> keys;
  // bv_keyswitch.cpp:92-98
  const BvKeySwitchKey &get(uint32_t galois_k) const {
    for (const auto &k : keys)
      if (k.galois_k == galois_k) return k;
    throw std::out_of_range("BvGaloisKeys::get: galois_k not found");
  }
};
}  // namespace bvks

// pir_session.h:8-18
struct PirSessionKeys {
  bvks::BvGaloisKeys bv_galois_keys;
  GSWCt gsw_key;
};
using SharedPirSessionKeys = std::shared_ptr<const PirSessionKeys>;

// pir.h:35-39 and 46-50
struct PirLayoutConfig {
  size_t target_num_pt;
  size_t expansion_height;
  bool fst_dim_pow2;
};
struct PirQueryShapeConfig {
  size_t fst_dim_sz;
  size_t num_selector_bits;
  size_t expansion_height;
};

// server.h:13
using PlaintextSource = std::function<void(size_t logical_index, RlwePt &out)>;

namespace detail {
[[noreturn]] inline void raise(opir_status st, const std::string &msg) {
  switch (st) {
    case OPIR_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    case OPIR_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
    case OPIR_ERR_OVERFLOW: throw std::overflow_error(msg);
    case OPIR_ERR_NO_MEMORY: throw std::bad_alloc();
    default: throw std::runtime_error(msg);
  }
}
inline void check(opir_status st, const char *what) {
  if (st != OPIR_OK) raise(st, std::string(what) + " failed (status " + std::to_string(st) + ")");
}
}  // namespace detail

// ------------------------------------------------------------- parameters
// PirParams (pir.h:53-167) of one parameter set. The default constructor is
// the library's default layout of CONFIG_N2048_K1_COMP; with_layout gives
// any other layout of the same set.
class PirParams {
 public:
  explicit PirParams(opir_config config = OPIR_CONFIG_N2048_K1_COMP)
      : PirParams(config, PirLayoutConfig{43690, 10, true}) {}
  PirParams(opir_config config, const PirLayoutConfig &layout) : config_(config) {
    const opir_layout l{layout.target_num_pt, static_cast<uint32_t>(layout.expansion_height),
                        layout.fst_dim_pow2 ? 1u : 0u};
    detail::check(opir_params_init_config(config, &l, &p_), "PirParams::with_layout");
  }

  PirParams with_layout(const PirLayoutConfig &layout) const { return PirParams(config_, layout); }
  PirParams with_query_shape(const PirQueryShapeConfig &shape) const {
    const opir_query_shape s{shape.fst_dim_sz, static_cast<uint32_t>(shape.num_selector_bits),
                             static_cast<uint32_t>(shape.expansion_height)};
    PirParams out(*this);
    detail::check(opir_params_query_shape(&p_, &s, &out.p_), "PirParams::with_query_shape");
    return out;
  }

  size_t get_num_pt() const { return p_.num_pt; }
  size_t get_target_num_pt() const { return p_.target_num_pt; }
  size_t get_num_dims() const { return p_.num_dims; }
  size_t get_num_other_dims() const { return p_.num_dims - 1; }
  size_t get_l() const { return p_.l_ep; }
  size_t get_l_key() const { return p_.l_key; }
  size_t get_small_q() const { return p_.small_q; }
  size_t get_base_log2() const { return p_.base_log2; }
  size_t get_base_log2_key() const { return p_.base_log2_key; }
  size_t get_fst_dim_sz() const { return p_.fst_dim_sz; }
  size_t get_other_dim_sz() const { return p_.num_pt / p_.fst_dim_sz; }
  size_t get_expan_height() const { return p_.expansion_height; }
  bool get_fst_dim_pow2() const { return p_.fst_dim_pow2 != 0; }
  size_t get_poly_degree() const { return p_.poly_degree; }
  uint64_t get_plain_mod() const { return p_.plain_mod; }
  size_t get_ct_mod_width() const { return p_.ct_mod_width; }
  // the logical modulus q (K = 1) or the two RNS limbs (K = 2)
  std::vector<uint64_t> get_rns_mods() const {
    return K() == 1 ? std::vector<uint64_t>{p_.q} : std::vector<uint64_t>{p_.q1, p_.q2};
  }
  size_t K() const { return p_.num_limbs; }
  size_t get_coeff_val_cnt() const { return static_cast<size_t>(p_.poly_degree) * K(); }
  size_t get_num_bits_per_coeff() const {
    size_t bits = 0;
    while ((1ull << (bits + 1)) <= p_.plain_mod) ++bits;
    return bits;
  }
  size_t get_pt_size() const { return get_num_bits_per_coeff() * p_.poly_degree / 8; }
  double get_DBSize_MB() const { return static_cast<double>(p_.num_pt) * get_pt_size() / 1024 / 1024; }
  // pir.h:115-139 (communication models only)
  size_t get_BFV_size(bool use_seed = true) const {
    return use_seed ? 32 + get_ct_mod_width() * p_.poly_degree / 8
                    : get_ct_mod_width() * p_.poly_degree * 2 / 8;
  }
  size_t get_gsw_key_size(bool use_seed = true) const { return 2 * p_.l_key * get_BFV_size(use_seed); }
  size_t get_bv_galois_key_size(bool use_seed = true) const {
    const size_t per_poly = (p_.poly_degree * get_ct_mod_width() + 7) / 8;
    return use_seed ? p_.expansion_height * p_.l_ks * (per_poly + 32)
                    : p_.expansion_height * p_.l_ks * 2 * per_poly;
  }

  const opir_params &raw() const { return p_; }
  opir_config config() const { return config_; }

 private:
  opir_config config_;
  opir_params p_{};
};

// ------------------------------------------------------------- server
// PirServer (server.h:15-172) backed by one device handle.
class PirServer {
 public:
  explicit PirServer(const PirParams &pir_params, int device = 0) : params_(pir_params) {
    opir_server *h = nullptr;
    detail::check(opir_server_create(&pir_params.raw(), device, &h), "PirServer::PirServer");
    h_.reset(h);
  }

  const PirParams &get_params() const { return params_; }

  // server.cpp:80-203. The source is called once per logical index, in
  // order; the plaintexts at record_indices (the zero padding too) are kept
  // for direct_get_original_plaintext.
  void load_data(size_t logical_num_pt, const PlaintextSource &source,
                 const std::vector<size_t> &record_indices = {}) {
    if (!source) throw std::invalid_argument("PirServer::load_data requires a source");
    for (size_t i : record_indices)
      if (i >= params_.get_num_pt())
        throw std::invalid_argument("PirServer::load_data record index exceeds its layout");
    Loader ld{this, &source, {}, {}, nullptr};
    for (size_t i : record_indices) ld.record.emplace(i, true);
    recorded_pts_.clear();
    const opir_status st = opir_server_load_db_source(h_.get(), logical_num_pt, &Loader::call, &ld);
    if (ld.error) std::rethrow_exception(ld.error);
    status(st, "PirServer::load_data");
    for (size_t i : record_indices)
      if (i >= logical_num_pt) recorded_pts_[i].data.assign(params_.get_poly_degree(), 0);
  }

  // server.cpp:53-66: a random database (uniform coefficients < t).
  void gen_data(const std::vector<size_t> &record_indices = {}) {
    std::mt19937_64 rng(std::random_device{}());
    const uint64_t t = params_.get_plain_mod();
    load_data(params_.get_num_pt(), [&](size_t, RlwePt &pt) {
      pt.data.resize(params_.get_poly_degree());
      for (auto &c : pt.data) c = rng() % t;
    }, record_indices);
  }

  // server.cpp:857-875
  void set_client_bv_galois_key(const size_t client_id, bvks::BvGaloisKeys bv_keys) {
    pending_bv_[client_id] = std::move(bv_keys);
    push_keys(client_id);
  }
  void set_client_gsw_key(const size_t client_id, GSWCt gsw_key) {
    pending_gsw_[client_id] = std::move(gsw_key);
    push_keys(client_id);
  }
  void set_client_session_keys(size_t client_id, SharedPirSessionKeys keys) {
    if (!keys) throw std::invalid_argument("PirServer session key bundle cannot be null");
    upload_keys(client_id, keys->bv_galois_keys, keys->gsw_key);
    sessions_[client_id] = std::move(keys);
  }
  SharedPirSessionKeys client_session_keys(size_t client_id) const {
    return sessions_.at(client_id);
  }

  // server.cpp:895-947
  RlweCt make_query(const size_t client_id, RlweCt &query) {
    const std::vector<uint64_t> q = flat(query);
    std::vector<uint64_t> resp(2 * params_.get_poly_degree());
    status(opir_server_make_query(h_.get(), client_id, q.data(), resp.data()),
           "PirServer::make_query");
    return unflat(resp.data(), params_.get_poly_degree(), false);
  }
  // Batched form (no counterpart in the reference): n queries in one pass.
  std::vector<RlweCt> make_query_batch(const std::vector<size_t> &client_ids,
                                       std::vector<RlweCt> &queries) {
    if (client_ids.size() != queries.size())
      throw std::invalid_argument("make_query_batch: one client id per query");
    std::vector<uint64_t> ids(client_ids.begin(), client_ids.end()), q;
    for (auto &ct : queries) {
      const auto f = flat(ct);
      q.insert(q.end(), f.begin(), f.end());
    }
    const size_t n = queries.size(), per = 2 * params_.get_poly_degree();
    std::vector<uint64_t> resp(n * per);
    status(opir_server_make_query_batch(h_.get(), static_cast<uint32_t>(n), ids.data(), q.data(),
                                        resp.data()),
           "PirServer::make_query_batch");
    std::vector<RlweCt> out;
    for (size_t i = 0; i < n; ++i)
      out.push_back(unflat(resp.data() + i * per, params_.get_poly_degree(), false));
    return out;
  }

  // server.cpp:818-821
  std::vector<RlweCt> expand_query(size_t client_id, RlweCt &query) const {
    const std::vector<uint64_t> q = flat(query);
    const size_t useful = params_.get_fst_dim_sz() + params_.get_l() * params_.get_num_other_dims();
    std::vector<uint64_t> out(useful * ct_words());
    status(opir_server_expand_query(h_.get(), client_id, q.data(), out.data()),
           "PirServer::expand_query");
    return unflat_many(out, useful, false);
  }
  // server.cpp:823-855
  std::vector<GSWCt> complete_selectors(size_t client_id, const std::vector<RlweCt> &expanded) {
    std::vector<uint64_t> in;
    for (const auto &ct : expanded) {
      const auto f = flat(ct);
      in.insert(in.end(), f.begin(), f.end());
    }
    const size_t nsel = params_.get_num_other_dims(), rows = 2 * params_.get_l();
    std::vector<uint64_t> out(std::max<size_t>(nsel, 1) * rows * ct_words());
    status(opir_server_complete_selectors(h_.get(), client_id, in.data(), out.data()),
           "PirServer::complete_selectors");
    std::vector<GSWCt> sel(nsel);
    for (size_t s = 0; s < nsel; ++s)
      for (size_t r = 0; r < rows; ++r) {
        const uint64_t *row = out.data() + (s * rows + r) * ct_words();
        sel[s].emplace_back(row, row + ct_words());
      }
    return sel;
  }
  // server.cpp:313-405
  std::vector<RlweCt> evaluate_first_dim(std::vector<RlweCt> &selection_vector) {
    std::vector<uint64_t> in;
    for (size_t i = 0; i < params_.get_fst_dim_sz() && i < selection_vector.size(); ++i) {
      const auto f = flat(selection_vector[i]);
      in.insert(in.end(), f.begin(), f.end());
    }
    if (in.size() != params_.get_fst_dim_sz() * ct_words())
      throw std::invalid_argument("evaluate_first_dim: fewer selection ciphertexts than fst_dim_sz");
    const size_t other = params_.get_other_dim_sz();
    std::vector<uint64_t> out(other * ct_words());
    status(opir_server_evaluate_first_dim(h_.get(), in.data(), out.data()),
           "PirServer::evaluate_first_dim");
    return unflat_many(out, other, false);
  }
  // server.cpp:599-649
  RlweCt evaluate_other_dim(std::vector<RlweCt> &intermediate_db, std::vector<GSWCt> &selectors) {
    std::vector<uint64_t> mid, sel;
    for (const auto &ct : intermediate_db) {
      const auto f = flat(ct);
      mid.insert(mid.end(), f.begin(), f.end());
    }
    for (const auto &g : selectors)
      for (const auto &row : g) sel.insert(sel.end(), row.begin(), row.end());
    if (sel.empty()) sel.push_back(0);
    std::vector<uint64_t> out(ct_words());
    status(opir_server_evaluate_other_dim(h_.get(), mid.data(), sel.data(), out.data()),
           "PirServer::evaluate_other_dim");
    return unflat(out.data(), params_.get_coeff_val_cnt(), false);
  }
  // server.cpp:652-722: result = x + b (y - x). Unlike the reference, y is
  // left as it was (callers do not read it afterwards).
  void ext_prod_mux(RlweCt &x, RlweCt &y, GSWCt &selection_cipher, RlweCt &result) {
    const auto fx = flat(x), fy = flat(y);
    std::vector<uint64_t> sel;
    for (const auto &row : selection_cipher) sel.insert(sel.end(), row.begin(), row.end());
    if (sel.size() != 2 * params_.get_l() * ct_words())
      throw std::invalid_argument("ext_prod_mux: selector must hold 2 L_EP rows");
    std::vector<uint64_t> out(ct_words());
    status(opir_server_ext_prod_mux(h_.get(), fx.data(), fy.data(), sel.data(), out.data()),
           "PirServer::ext_prod_mux");
    result = unflat(out.data(), params_.get_coeff_val_cnt(), false);
  }

  // server.cpp:950-1009
  size_t save_resp_to_stream(const RlweCt &response, std::stringstream &resp_stream) {
    const size_t n = params_.get_poly_degree();
    if (response.c0.size() != n || response.c1.size() != n)
      throw std::invalid_argument("save_resp_to_stream: response must hold N coefficients per polynomial");
    std::vector<uint64_t> r(2 * n);
    std::copy(response.c0.begin(), response.c0.end(), r.begin());
    std::copy(response.c1.begin(), response.c1.end(), r.begin() + n);
    std::vector<uint8_t> bytes(opir_response_bytes(&params_.raw()));
    const size_t got = opir_save_response(&params_.raw(), r.data(), bytes.data(), bytes.size());
    resp_stream.write(reinterpret_cast<const char *>(bytes.data()), static_cast<std::streamsize>(got));
    return got;
  }

  // server.cpp:885-893 (test helper): a plaintext recorded at load time.
  RlwePt direct_get_original_plaintext(const size_t index) const {
    auto it = recorded_pts_.find(index);
    if (it == recorded_pts_.end())
      throw std::invalid_argument("Plaintext index " + std::to_string(index) +
                                  " was not recorded during database loading");
    return it->second;
  }

  opir_server *handle() const { return h_.get(); }

 private:
  struct Deleter {
    void operator()(opir_server *s) const { opir_server_destroy(s); }
  };
  struct Loader {
    PirServer *self;
    const PlaintextSource *source;
    std::unordered_map<size_t, bool> record;
    RlwePt pt;
    std::exception_ptr error;
    static int call(void *user, uint64_t idx, uint64_t *out) {
      auto *ld = static_cast<Loader *>(user);
      try {
        ld->pt.data.clear();
        (*ld->source)(static_cast<size_t>(idx), ld->pt);
        const size_t n = ld->self->params_.get_poly_degree();
        if (ld->pt.data.size() != n)
          throw std::invalid_argument("Plaintext source returned the wrong coefficient count");
        std::copy(ld->pt.data.begin(), ld->pt.data.end(), out);
        if (ld->record.count(static_cast<size_t>(idx))) ld->self->recorded_pts_[idx] = ld->pt;
        return 0;
      } catch (...) {
        ld->error = std::current_exception();
        return 1;
      }
    }
  };

  void status(opir_status st, const char *what) const {
    if (st == OPIR_OK) return;
    const char *msg = opir_server_last_error(h_.get());
    detail::raise(st, std::string(what) + ": " + (msg ? msg : ""));
  }
  size_t ct_words() const { return 2 * params_.get_coeff_val_cnt(); }
  std::vector<uint64_t> flat(const RlweCt &ct) const {
    const size_t n = params_.get_coeff_val_cnt();
    if (ct.c0.size() != n || ct.c1.size() != n)
      throw std::invalid_argument("ciphertext must hold K*N coefficients per polynomial");
    if (ct.ntt_form) throw std::invalid_argument("ciphertext must be in coefficient form");
    std::vector<uint64_t> f(2 * n);
    std::copy(ct.c0.begin(), ct.c0.end(), f.begin());
    std::copy(ct.c1.begin(), ct.c1.end(), f.begin() + n);
    return f;
  }
  static RlweCt unflat(const uint64_t *p, size_t n, bool ntt) {
    RlweCt ct;
    ct.c0.assign(p, p + n);
    ct.c1.assign(p + n, p + 2 * n);
    ct.ntt_form = ntt;
    return ct;
  }
  std::vector<RlweCt> unflat_many(const std::vector<uint64_t> &v, size_t count, bool ntt) const {
    std::vector<RlweCt> out;
    for (size_t i = 0; i < count; ++i)
      out.push_back(unflat(v.data() + i * ct_words(), params_.get_coeff_val_cnt(), ntt));
    return out;
  }
  // The C ABI takes a client's BV and RGSW keys together: a client is
  // registered once both halves are present.
  void push_keys(size_t client_id) {
    auto b = pending_bv_.find(client_id);
    auto g = pending_gsw_.find(client_id);
    if (b == pending_bv_.end() || g == pending_gsw_.end()) return;
    upload_keys(client_id, b->second, g->second);
  }
  void upload_keys(size_t client_id, const bvks::BvGaloisKeys &bv, const GSWCt &gsw) {
    const size_t kn = params_.get_coeff_val_cnt();
    std::vector<uint64_t> rows;
    std::vector<uint32_t> ks;
    for (const auto &key : bv.keys) {
      ks.push_back(key.galois_k);
      for (const auto &ct : key.cts) {
        if (ct.a.size() != kn || ct.b.size() != kn)
          throw std::invalid_argument("BV key polynomial must hold K*N coefficients");
        rows.insert(rows.end(), ct.b.begin(), ct.b.end());
        rows.insert(rows.end(), ct.a.begin(), ct.a.end());
      }
      if (key.cts.size() != params_.raw().l_ks)
        throw std::invalid_argument("BV key switching key must hold L_KS ciphertexts");
    }
    std::vector<uint64_t> g;
    for (const auto &row : gsw) {
      if (row.size() != 2 * kn) throw std::invalid_argument("RGSW row must hold 2*K*N coefficients");
      g.insert(g.end(), row.begin(), row.end());
    }
    if (gsw.size() != 2 * params_.get_l_key())
      throw std::invalid_argument("RGSW key must hold 2 L_KEY rows");
    if (rows.empty()) rows.push_back(0);
    if (ks.empty()) ks.push_back(0);
    status(opir_server_set_client_keys(h_.get(), client_id, rows.data(), ks.data(),
                                       static_cast<uint32_t>(bv.keys.size()), g.data()),
           "PirServer::set_client_keys");
  }

  PirParams params_;
  std::unique_ptr<opir_server, Deleter> h_;
  std::map<size_t, bvks::BvGaloisKeys> pending_bv_;
  std::map<size_t, GSWCt> pending_gsw_;
  std::map<size_t, SharedPirSessionKeys> sessions_;
  std::unordered_map<size_t, RlwePt> recorded_pts_;
};

// ------------------------------------------------------------- client
// The GPU forms of PirClient's steps that scale with queries, responses and
// sessions (client.cpp:25-225, 364-410) for one client's secret. The
// randomness the reference client draws from its own generators (each
// query's uniform c1 and error, each key row's uniform part and error) is
// passed in, so results equal the reference client's for the same draws.
class GpuPirClient {
 public:
  // secret: the coefficient form of the client's RlweSk, N values in {-1, 0, 1}.
  GpuPirClient(const PirParams &pir_params, const std::vector<int8_t> &secret, int device = 0)
      : params_(pir_params) {
    if (secret.size() != pir_params.get_poly_degree())
      throw std::invalid_argument("GpuPirClient: the secret holds N coefficients");
    opir_client *h = nullptr;
    detail::check(opir_client_create(&pir_params.raw(), secret.data(), device, &h),
                  "GpuPirClient::GpuPirClient");
    h_.reset(h);
  }

  // fast_generate_query (client.cpp:107-225): c1 = a (K*N, limb-major),
  // c0 = -(a s + e) plus the packed plaintext.
  RlweCt fast_generate_query(size_t pt_idx, const std::vector<uint64_t> &a,
                             const std::vector<int64_t> &e) {
    return std::move(fast_generate_queries({pt_idx}, a, e).front());
  }
  // n queries at once: a is n x K*N, e is n x N.
  std::vector<RlweCt> fast_generate_queries(const std::vector<size_t> &pt_idx,
                                            const std::vector<uint64_t> &a,
                                            const std::vector<int64_t> &e) {
    const size_t n = pt_idx.size(), kn = params_.get_coeff_val_cnt();
    if (a.size() != n * kn || e.size() != n * params_.get_poly_degree())
      throw std::invalid_argument("GpuPirClient: a holds n x K*N and e n x N values");
    const std::vector<uint64_t> idx(pt_idx.begin(), pt_idx.end());
    std::vector<uint64_t> q(std::max<size_t>(1, n * 2 * kn));
    status(opir_client_generate_queries(h_.get(), static_cast<uint32_t>(n), idx.data(), a.data(),
                                        e.data(), q.data()),
           "GpuPirClient::fast_generate_query");
    std::vector<RlweCt> out(n);
    for (size_t i = 0; i < n; ++i) {
      out[i].c0.assign(q.begin() + i * 2 * kn, q.begin() + i * 2 * kn + kn);
      out[i].c1.assign(q.begin() + i * 2 * kn + kn, q.begin() + (i + 1) * 2 * kn);
    }
    return out;
  }

  // decrypt_mod_q (client.cpp:364-410) of a response as
  // load_resp_from_stream yields it (2 x N values below small_q).
  RlwePt decrypt_mod_q(const RlweCt &ct) { return std::move(decrypt_mod_q_batch({ct}).front()); }
  // n responses; *max_noise (optional) receives each one's max noise, the
  // figure the reference prints as its noise budget (client.cpp:389-407).
  std::vector<RlwePt> decrypt_mod_q_batch(const std::vector<RlweCt> &cts,
                                          std::vector<uint64_t> *max_noise = nullptr) {
    const size_t n = cts.size(), N = params_.get_poly_degree();
    std::vector<uint64_t> in(std::max<size_t>(1, n * 2 * N)), pt(std::max<size_t>(1, n * N));
    for (size_t i = 0; i < n; ++i) {
      if (cts[i].c0.size() != N || cts[i].c1.size() != N)
        throw std::invalid_argument("GpuPirClient: a response holds 2 x N values");
      std::copy(cts[i].c0.begin(), cts[i].c0.end(), in.begin() + i * 2 * N);
      std::copy(cts[i].c1.begin(), cts[i].c1.end(), in.begin() + i * 2 * N + N);
    }
    if (max_noise) max_noise->assign(std::max<size_t>(1, n), 0);
    status(opir_client_decrypt(h_.get(), static_cast<uint32_t>(n), in.data(), pt.data(),
                               max_noise ? max_noise->data() : nullptr),
           "GpuPirClient::decrypt_mod_q");
    if (max_noise) max_noise->resize(n);
    std::vector<RlwePt> out(n);
    for (size_t i = 0; i < n; ++i) out[i].data.assign(pt.begin() + i * N, pt.begin() + (i + 1) * N);
    return out;
  }

  // create_session_keys (client.cpp:40-45): the BV keys for galois_k =
  // N/2^i + 1, i < h (bv_a h*L_KS x K*N, bv_e h*L_KS x N) and RGSW(s)
  // (gsw_a 2 L_KEY x K*N, gsw_e 2 L_KEY x N), NTT form.
  PirSessionKeys create_session_keys(const std::vector<uint64_t> &bv_a,
                                     const std::vector<int64_t> &bv_e,
                                     const std::vector<uint64_t> &gsw_a,
                                     const std::vector<int64_t> &gsw_e) {
    const opir_params &p = params_.raw();
    const size_t kn = params_.get_coeff_val_cnt(), N = params_.get_poly_degree();
    const size_t bv_rows = static_cast<size_t>(p.expansion_height) * p.l_ks;
    const size_t gsw_rows = 2ull * p.l_key;
    if (bv_a.size() != bv_rows * kn || bv_e.size() != bv_rows * N ||
        gsw_a.size() != gsw_rows * kn || gsw_e.size() != gsw_rows * N)
      throw std::invalid_argument("GpuPirClient: key randomness of the wrong size");
    std::vector<uint64_t> bv(std::max<size_t>(1, bv_rows * 2 * kn)), g(gsw_rows * 2 * kn);
    status(opir_client_keygen(h_.get(), bv_rows ? bv_a.data() : nullptr,
                              bv_rows ? bv_e.data() : nullptr, gsw_a.data(), gsw_e.data(),
                              bv_rows ? bv.data() : nullptr, g.data()),
           "GpuPirClient::create_session_keys");
    PirSessionKeys keys;
    for (uint32_t i = 0; i < p.expansion_height; ++i) {
      bvks::BvKeySwitchKey key;
      key.galois_k = (p.poly_degree >> i) + 1;
      for (uint32_t r = 0; r < p.l_ks; ++r) {
        const auto row = bv.begin() + (static_cast<size_t>(i) * p.l_ks + r) * 2 * kn;
        key.cts.push_back(bvks::BvRlweCt{std::vector<uint64_t>(row + kn, row + 2 * kn),
                                         std::vector<uint64_t>(row, row + kn)});
      }
      keys.bv_galois_keys.keys.push_back(std::move(key));
    }
    for (size_t r = 0; r < gsw_rows; ++r)
      keys.gsw_key.emplace_back(g.begin() + r * 2 * kn, g.begin() + (r + 1) * 2 * kn);
    return keys;
  }

 private:
  struct Deleter {
    void operator()(opir_client *h) const { opir_client_destroy(h); }
  };
  void status(opir_status st, const char *what) const {
    if (st != OPIR_OK)
      detail::raise(st, std::string(what) + ": " + opir_client_last_error(h_.get()));
  }

  PirParams params_;
  std::unique_ptr<opir_client, Deleter> h_;
};

}  // namespace onionpir_b200
