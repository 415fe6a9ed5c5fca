// Host orchestration of the query paths whose limbs are 64-bit words: the
// PirServer methods (src/server.cpp) under CONFIG_N4096_K2_MP (two 60-bit
// limbs at N = 4096, the kernels of opir_c4_kernels.cu) and under
// CONFIG_N2048_K1 (one 60-bit prime at N = 2048, opir_k1p_kernels.cu); both
// share the 64-bit-limb tensor-core scan (opir_c4_scan_tc.cu). Every
// arithmetic step runs on the device; the host only validates inputs, moves
// buffers and enqueues launches on the handle's stream.
#include "opir_c4_server.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

#include "opir_k1p_kernels.h"
#include "opir_params.h"
#include "opir_scan_tc.h"

namespace opir4 {

using opir::ck;

namespace {

constexpr uint32_t kLKsRows = 8, kLKeyRows = 8;  // L_KS, L_KEY of both sets

// Appends one ciphertext-shaped row (2 N limbs u64, limb-major polynomials)
// and its Shoup companions floor(w 2^64 / q_limb) in the device row layout.
void append_row(std::vector<uint64_t> &dst, const uint64_t *row, uint32_t n, uint32_t limbs) {
  const uint64_t ct = 2ull * n * limbs;
  dst.insert(dst.end(), row, row + ct);
  for (uint64_t j = 0; j < ct; ++j) {
    const uint64_t q = (limbs == 2 && ((j / n) & 1)) ? kQ1 : kQ0;
    dst.push_back(static_cast<uint64_t>((static_cast<unsigned __int128>(row[j]) << 64) / q));
  }
}

uint32_t resp_bytes_of(const opir_params &p) {
  return static_cast<uint32_t>((2ull * p.poly_degree * p.small_q_width + 7) / 8);
}

Shape4 shape_of(const opir_params &p) {
  Shape4 s{};
  s.n0 = static_cast<uint32_t>(p.fst_dim_sz);
  s.n0p = static_cast<uint32_t>((p.fst_dim_sz + 15) / 16 * 16);
  s.other = static_cast<uint32_t>(p.other_dim_sz);
  s.num_dims = p.num_dims;
  s.h = p.expansion_height;
  s.useful = static_cast<uint32_t>(p.fst_dim_sz + static_cast<uint64_t>(p.l_ep) * (p.num_dims - 1));
  s.l_ep = p.l_ep;
  s.num_pt = p.num_pt;
  return s;
}

// Ciphertext slots per query of an expansion buffer: the widest tree level,
// the useful leaves, the padded first dimension and the candidate rows (the
// first dimension's query matrix, its byte planes and the scan's output
// reuse the two expansion buffers).
uint64_t lvl_slots_of(const Shape4 &s) {
  uint64_t slots = std::max<uint64_t>(1, std::max({s.useful, s.other, s.n0p}));
  for (uint32_t d = 0; d < s.h; ++d) slots = std::max<uint64_t>(slots, 2ull * expand_nodes(s, d));
  return slots;
}

struct Plan {
  size_t lvl, sel, mid, resp, keyptrs;
  uint64_t bytes() const { return (2 * lvl + sel + 2 * mid + resp) * 8 + keyptrs * sizeof(void *); }
};

// ct: u64 words per ciphertext (2 N limbs); row = 2 ct (with companions)
Plan plan_for(const Shape4 &s, uint64_t lvl_slots, uint32_t n, uint32_t N, uint64_t ct) {
  const uint64_t nsel = s.num_dims > 1 ? s.num_dims - 1 : 0;
  Plan pl{};
  pl.lvl = static_cast<size_t>(n) * lvl_slots * ct;
  pl.sel = std::max<uint64_t>(1, n * nsel * 2 * s.l_ep * 2 * ct);
  pl.mid = static_cast<size_t>(n) * s.other * ct;
  pl.resp = static_cast<size_t>(n) * 2 * N;
  pl.keyptrs = 2ull * n;
  return pl;
}

}  // namespace

opir_params derive(const opir_layout &layout) { return opir::derive_params_c4(layout); }

Server::Server(const opir_params &p, cudaStream_t stream, const opir::RowShard *rs)
    : p_(p), st_(stream) {
  k1_ = p_.num_limbs == 1;
  if (k1_ && (p_.poly_degree != static_cast<uint32_t>(opir1::kN) || p_.q != opir1::kQ))
    throw std::invalid_argument("unexpected CONFIG_N2048_K1 modulus");
  n_ = p_.poly_degree;
  limbs_ = p_.num_limbs;
  ct_ = 2ull * n_ * limbs_;
  row_ = 2 * ct_;
  out_words_ = 2ull * n_;
  sh_ = shape_of(p_);
  tree_h_ = sh_.num_dims > 1 ? sh_.num_dims - 1 : 0;
  if (rs) {
    tree_h_ = rs->tree_h;
    num_shards_ = rs->num_shards;
    host_rows_ = rs->rows;
    sh_.other = static_cast<uint32_t>(rs->rows.size());
    sh_.num_pt = static_cast<uint64_t>(sh_.other) * sh_.n0;
    out_words_ = ct_;
    shard_ = true;
    row_map_.alloc(rs->rows.size());
    ck(cudaMemcpy(row_map_.p, rs->rows.data(), rs->rows.size() * 4, cudaMemcpyHostToDevice),
       "row map");
  }
  lvl_slots_ = lvl_slots_of(sh_);
  if (k1_) {
    setup_k1_tables();
  } else {
    setup_c4_tables();
  }
  dp_.small_q = p_.small_q;
  dp_.small_q_width = p_.small_q_width;
  const uint64_t planes = static_cast<uint64_t>(n_) * limbs_ * 8;  // byte planes of the database
  const uint64_t db_bytes = planes * sh_.other * sh_.n0p;
  db8_.alloc(db_bytes);
  ck(cudaMemsetAsync(db8_.p, 0, db_bytes, st_), "db memset");
  opir::make_plane_map(&map_db_, db8_.p, sh_.n0p, sh_.other, planes, 128, 64);
  err_.alloc(1);
  ck(cudaMemsetAsync(err_.p, 0, sizeof(uint32_t), st_), "err memset");
  progress_.alloc(1024);  // one counter per scan CTA (the grid is at most the SM count)
  int dev = 0;
  ck(cudaGetDevice(&dev), "device");
  ck(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev), "sm count");
  if (const char *g = std::getenv("OPIR_GRAPHS")) use_graphs_ = std::strcmp(g, "0") != 0;
  ck(cudaStreamSynchronize(st_), "create");
}

// Twiddle tables of CONFIG_N2048_K1: [forward N][inverse N] (w, Shoup) of
// the one limb, the first 64 of each to constant memory.
void Server::setup_k1_tables() {
  const opir::LimbTables64 t = opir::make_limb_tables64(n_, p_.q, p_.w1);
  // [forward N][inverse N] (w, Shoup) pairs, then (psi^m, Shoup) for m < 2N
  std::vector<ulonglong2> host(4ull * n_);
  for (uint32_t i = 0; i < n_; ++i) {
    host[i] = make_ulonglong2(t.fw[i], t.fw_sh[i]);
    host[n_ + i] = make_ulonglong2(t.iw[i], t.iw_sh[i]);
  }
  {
    // psi = fw[brev(1)] = fw[N / 2] (fw[k] = psi^brev(k))
    const uint64_t q = t.q, psi = t.fw[n_ / 2];
    uint64_t pw = 1;
    for (uint32_t m = 0; m < 2 * n_; ++m) {
      const uint64_t sh = static_cast<uint64_t>((static_cast<unsigned __int128>(pw) << 64) / q);
      host[2 * n_ + m] = make_ulonglong2(pw, sh);
      pw = static_cast<uint64_t>(static_cast<unsigned __int128>(pw) * psi % q);
    }
    if (pw != 1 || host[2 * n_ + n_].x != q - 1)
      throw std::runtime_error("psi is not a primitive 2N-th root of unity");
  }
  tables_.alloc(host.size());
  ck(cudaMemcpy(tables_.p, host.data(), host.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice),
     "twiddle tables");
  dp_.T.fwt[0] = dp_.T.fwt[1] = tables_.p;
  dp_.T.iwt[0] = dp_.T.iwt[1] = tables_.p + n_;
  dp_.T.pwt[0] = dp_.T.pwt[1] = tables_.p + 2 * n_;
  const uint64_t ninv[2] = {t.n_inv, t.n_inv_sh}, w1n[2] = {t.w1_ninv, t.w1_ninv_sh};
  opir1::upload_constants(t.fw.data(), t.fw_sh.data(), t.iw.data(), t.iw_sh.data(), ninv, w1n);
}

opir1::Dev1 Server::d1() const {
  return opir1::Dev1{dp_.T.fwt[0], dp_.T.iwt[0], dp_.small_q, dp_.small_q_width, dp_.T.pwt[0]};
}

// Twiddle tables of CONFIG_N4096_K2_MP: [limb][forward N][inverse N].
void Server::setup_c4_tables() {
  const opir::LimbTables64 t[2] = {opir::make_limb_tables64(kN, p_.q1, p_.w1),
                                   opir::make_limb_tables64(kN, p_.q2, p_.w2)};
  if (t[0].q != kQ0 || t[1].q != kQ1) throw std::invalid_argument("unexpected RNS limbs");
  // [limb][forward N][inverse N] (w, Shoup) pairs, then [limb][psi^m, m < 2N]
  std::vector<ulonglong2> host(8ull * kN);
  for (int l = 0; l < 2; ++l) {
    for (int i = 0; i < kN; ++i) {
      host[l * 2 * kN + i] = make_ulonglong2(t[l].fw[i], t[l].fw_sh[i]);
      host[l * 2 * kN + kN + i] = make_ulonglong2(t[l].iw[i], t[l].iw_sh[i]);
    }
    // psi = fw[brev(1)] = fw[N / 2] (fw[k] = psi^brev(k))
    const uint64_t q = t[l].q, psi = t[l].fw[kN / 2];
    uint64_t pw = 1;
    for (int m = 0; m < 2 * kN; ++m) {
      const uint64_t sh = static_cast<uint64_t>((static_cast<unsigned __int128>(pw) << 64) / q);
      host[4 * kN + l * 2 * kN + m] = make_ulonglong2(pw, sh);
      pw = static_cast<uint64_t>(static_cast<unsigned __int128>(pw) * psi % q);
    }
    if (pw != 1 || host[4 * kN + l * 2 * kN + kN].x != q - 1)
      throw std::runtime_error("psi is not a primitive 2N-th root of unity");
  }
  tables_.alloc(host.size());
  ck(cudaMemcpy(tables_.p, host.data(), host.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice),
     "twiddle tables");
  for (int l = 0; l < 2; ++l) {
    dp_.T.fwt[l] = tables_.p + l * 2 * kN;
    dp_.T.iwt[l] = tables_.p + l * 2 * kN + kN;
    dp_.T.pwt[l] = tables_.p + 4 * kN + l * 2 * kN;
  }
  const uint64_t *fw[2] = {t[0].fw.data(), t[1].fw.data()};
  const uint64_t *fw_sh[2] = {t[0].fw_sh.data(), t[1].fw_sh.data()};
  const uint64_t *iw[2] = {t[0].iw.data(), t[1].iw.data()};
  const uint64_t *iw_sh[2] = {t[0].iw_sh.data(), t[1].iw_sh.data()};
  const uint64_t ninv[2][2] = {{t[0].n_inv, t[0].n_inv_sh}, {t[1].n_inv, t[1].n_inv_sh}};
  const uint64_t w1n[2][2] = {{t[0].w1_ninv, t[0].w1_ninv_sh}, {t[1].w1_ninv, t[1].w1_ninv_sh}};
  upload_constants(fw, fw_sh, iw, iw_sh, ninv, w1n);
  dp_.q0inv = p_.q1_inv_mod_q2;
  dp_.q0inv_sh = static_cast<uint64_t>((static_cast<unsigned __int128>(dp_.q0inv) << 64) / kQ1);
}

// ------------------------------------------------------------------ launches
// The kernels of this handle's parameter set.
void Server::run_db_preprocess(const uint64_t *coeffs, uint64_t coeff_pt_begin, uint64_t seed,
                               uint64_t logical, uint64_t pb, uint64_t pe) {
  if (k1_)
    opir1::launch_db_preprocess(d1(), sh_, coeffs, coeff_pt_begin, seed, p_.plain_mod, logical, pb,
                                pe, db8_.p, st_);
  else
    launch_db_preprocess(dp_, sh_, coeffs, coeff_pt_begin, seed, p_.plain_mod, logical, pb, pe,
                         row_map_.p, db8_.p, st_);
}
void Server::run_selectors(const uint64_t *leaves, const uint64_t *const *gsw, uint32_t n) {
  if (k1_) opir1::launch_selectors(d1(), sh_, leaves, lvl_slots_, gsw, sel_.p, n, st_);
  else launch_selectors(dp_, sh_, leaves, lvl_slots_, gsw, sel_.p, n, st_);
}
void Server::run_mux(const Shape4 &sh, uint32_t level, uint32_t tree_h, const uint64_t *in,
                     uint64_t *out, uint64_t mid_stride, const uint64_t *sel, uint32_t n) {
  if (k1_) opir1::launch_mux_level(d1(), sh, level, tree_h, in, out, mid_stride, sel, n, st_);
  else launch_mux_level(dp_, sh, level, tree_h, in, out, mid_stride, sel, n, st_);
}
void Server::run_modswitch(const uint64_t *ct, uint64_t ct_stride, uint64_t *resp, uint32_t n) {
  if (k1_) opir1::launch_modswitch(d1(), ct, ct_stride, resp, nullptr, resp_bytes_of(p_), n, st_);
  else launch_modswitch(dp_, ct, ct_stride, resp, nullptr, resp_bytes_of(p_), n, st_);
}

Server::~Server() {
  if (st_) cudaStreamSynchronize(st_);
  clear_graphs();
  for (PtrSlot &sl : ring_) {
    if (sl.host) cudaFreeHost(sl.host);
    if (sl.done) cudaEventDestroy(sl.done);
  }
}

// ------------------------------------------------------------------ database
template <typename Fill>
void Server::load_tiles(uint64_t logical, Fill &&fill) {
  if (logical > p_.num_pt)
    throw std::invalid_argument("PirServer::load_data logical plaintext count exceeds its layout");
  const uint64_t local_pt = static_cast<uint64_t>(sh_.other) * sh_.n0;
  const uint64_t tile = 2048;
  std::vector<uint64_t> host(tile * n_);
  opir::DevBuf<uint64_t> dev;
  dev.alloc(tile * n_);
  db_loaded_ = false;
  for (uint64_t pb = 0; pb < local_pt; pb += tile) {
    const uint64_t pe = std::min<uint64_t>(local_pt, pb + tile);
    opir::fill_runs(host_rows_, sh_.n0, logical, pb, pe, host.data(), fill, n_);
    ck(cudaMemcpyAsync(dev.p, host.data(), (pe - pb) * n_ * 8, cudaMemcpyHostToDevice, st_),
       "db upload");
    run_db_preprocess(dev.p, pb, 0, logical, pb, pe);
    ck(cudaStreamSynchronize(st_), "db preprocess");
  }
  db_loaded_ = true;
}

void Server::load_db(uint64_t logical, const uint64_t *coeffs) {
  const uint64_t t = p_.plain_mod;
  load_tiles(logical, [&](uint64_t b, uint64_t e, uint64_t *dst) {
    const uint64_t *src = coeffs + b * n_;
    for (uint64_t i = 0; i < (e - b) * n_; ++i) {
      if (src[i] >= t)
        throw std::invalid_argument("Plaintext source coefficient exceeds the plaintext modulus");
      dst[i] = src[i];
    }
  });
}

void Server::load_db_u16(uint64_t logical, const uint16_t *coeffs) {
  const uint64_t t = p_.plain_mod;
  load_tiles(logical, [&](uint64_t b, uint64_t e, uint64_t *dst) {
    const uint16_t *src = coeffs + b * n_;
    for (uint64_t i = 0; i < (e - b) * n_; ++i) {
      if (src[i] >= t)
        throw std::invalid_argument("Plaintext source coefficient exceeds the plaintext modulus");
      dst[i] = src[i];
    }
  });
}

void Server::load_db_source(uint64_t logical, opir_plaintext_source source, void *user) {
  const uint64_t t = p_.plain_mod;
  load_tiles(logical, [&](uint64_t b, uint64_t e, uint64_t *dst) {
    for (uint64_t idx = b; idx < e; ++idx) {
      uint64_t *pt = dst + (idx - b) * n_;
      if (source(user, idx, pt) != 0) throw std::invalid_argument("Plaintext source failed");
      for (uint32_t c = 0; c < n_; ++c)
        if (pt[c] >= t)
          throw std::invalid_argument("Plaintext source coefficient exceeds the plaintext modulus");
    }
  });
}

void Server::load_db_seeded(uint64_t logical, uint64_t seed) {
  if (logical > p_.num_pt)
    throw std::invalid_argument("PirServer::load_data logical plaintext count exceeds its layout");
  db_loaded_ = false;
  const uint64_t chunk = 1ull << 18;
  const uint64_t local_pt = static_cast<uint64_t>(sh_.other) * sh_.n0;
  for (uint64_t pb = 0; pb < local_pt; pb += chunk)
    run_db_preprocess(nullptr, 0, seed, logical, pb, std::min<uint64_t>(local_pt, pb + chunk));
  ck(cudaStreamSynchronize(st_), "db preprocess");
  db_loaded_ = true;
}

// ------------------------------------------------------------------ clients
void Server::check_ct_values(const uint64_t *v, size_t cts) const {
  const uint32_t parts = 2 * limbs_;  // polynomial limbs of a ciphertext, limb-major
  for (size_t c = 0; c < cts; ++c)
    for (uint32_t part = 0; part < parts; ++part) {
      const uint64_t q = (limbs_ == 2 && (part & 1)) ? kQ1 : kQ0;
      const uint64_t *w = v + c * ct_ + static_cast<size_t>(part) * n_;
      for (uint32_t j = 0; j < n_; ++j)
        if (w[j] >= q) throw std::invalid_argument("ciphertext coefficient not reduced mod its limb");
    }
}

void Server::set_client_keys(uint64_t id, const uint64_t *bv_keys, const uint32_t *galois_ks,
                             uint32_t n_keys, const uint64_t *gsw_key) {
  const uint32_t h = p_.expansion_height;
  if (!gsw_key) throw std::invalid_argument("PirServer session key bundle cannot be null");
  if (n_keys < h) throw std::invalid_argument("PirServer session lacks keys for its expansion height");
  if (n_keys && (!bv_keys || !galois_ks)) throw std::invalid_argument("null BV key arrays");
  const size_t key_words = static_cast<size_t>(kLKsRows) * ct_;  // one BvKeySwitchKey
  std::vector<int> order(h);
  for (uint32_t d = 0; d < h; ++d) {
    const uint32_t want = n_ / (1u << d) + 1;
    order[d] = -1;
    for (uint32_t i = 0; i < n_keys; ++i)
      if (galois_ks[i] == want) { order[d] = static_cast<int>(i); break; }
    if (order[d] < 0) throw std::out_of_range("BvGaloisKeys::get: galois_k not found");
    check_ct_values(bv_keys + order[d] * key_words, kLKsRows);
  }
  const size_t gsw_rows = 2ull * kLKeyRows;
  check_ct_values(gsw_key, gsw_rows);
  // device rows carry their Shoup companions (opir_c4_kernels.h)
  std::vector<uint64_t> bv_rows, gsw_rows_host;
  bv_rows.reserve(static_cast<size_t>(h) * kLKsRows * row_);
  for (uint32_t d = 0; d < h; ++d)
    for (uint32_t r = 0; r < kLKsRows; ++r)
      append_row(bv_rows, bv_keys + order[d] * key_words + r * ct_, n_, limbs_);
  for (size_t r = 0; r < gsw_rows; ++r) append_row(gsw_rows_host, gsw_key + r * ct_, n_, limbs_);
  Keys k;
  k.bv.alloc(std::max<size_t>(1, bv_rows.size()));
  k.gsw.alloc(gsw_rows_host.size());
  if (!bv_rows.empty())
    ck(cudaMemcpyAsync(k.bv.p, bv_rows.data(), bv_rows.size() * 8, cudaMemcpyHostToDevice, st_),
       "bv upload");
  ck(cudaMemcpyAsync(k.gsw.p, gsw_rows_host.data(), gsw_rows_host.size() * 8,
                     cudaMemcpyHostToDevice, st_), "gsw upload");
  ck(cudaStreamSynchronize(st_), "key upload");
  Keys &slot = clients_[id];
  slot.bv.swap(k.bv);
  slot.gsw.swap(k.gsw);
}

void Server::remove_client(uint64_t id) {
  ck(cudaStreamSynchronize(st_), "remove_client");
  if (clients_.erase(id) == 0) throw std::out_of_range("unknown client id");
}

// ------------------------------------------------------------------ scratch
void Server::clear_graphs() {
  for (auto &kv : graphs_) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  graphs_.clear();
  graph_seen_.clear();
}

void Server::ensure_capacity(uint32_t n) {
  if (n <= cap_) return;
  clear_graphs();
  const Plan pl = plan_for(sh_, lvl_slots_, n, n_, ct_);
  for (auto &b : lvl_) b.alloc(pl.lvl);
  sel_.alloc(pl.sel);
  for (auto &b : mid_) b.alloc(pl.mid);
  resp_.alloc(static_cast<size_t>(n) * out_words_);
  q_in_.alloc(static_cast<size_t>(n) * ct_);
  keyptrs_.alloc(pl.keyptrs);
  cap_ = n;
}

void Server::reserve(uint32_t max_batch) {
  ensure_capacity(max_batch);
  grow_ptr_slots(2ull * max_batch);
}

void Server::plan_memory(const opir_params &p, opir_memory_plan *out) {
  const Shape4 s = shape_of(p);
  const uint64_t slots = lvl_slots_of(s);
  const uint32_t N = p.poly_degree;
  const uint64_t ct = 2ull * N * p.num_limbs;
  const uint64_t one = plan_for(s, slots, 1, N, ct).bytes(), two = plan_for(s, slots, 2, N, ct).bytes();
  out->database_bytes = static_cast<uint64_t>(N) * p.num_limbs * 8 * s.other * s.n0p +
                        2ull * N * p.num_limbs * sizeof(ulonglong2) + sizeof(uint32_t);
  out->client_key_bytes =
      (static_cast<uint64_t>(p.expansion_height) * kLKsRows + 2ull * kLKeyRows) * 2 * ct * 8;
  out->scratch_bytes_per_query = two - one;
  out->scratch_bytes_fixed = 2 * one - two;
}

void Server::grow_ptr_slots(size_t entries) {
  for (PtrSlot &sl : ring_) {
    if (!sl.done) ck(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "event");
    if (sl.cap >= entries) continue;
    ck(cudaEventSynchronize(sl.done), "key pointer slot");
    if (sl.host) cudaFreeHost(sl.host);
    sl.host = nullptr;
    sl.cap = 0;
    ck(cudaMallocHost(reinterpret_cast<void **>(&sl.host), entries * sizeof(void *)),
       "cudaMallocHost");
    sl.cap = entries;
  }
}

// Per-query key pointers (BV then RGSW) from a pinned slot of a small ring,
// so the upload is asynchronous; a slot is refilled only after the copy that
// last read it has run.
void Server::upload_keyptrs(const uint64_t *ids, uint32_t n) {
  host_ptrs_.resize(2ull * n);
  for (uint32_t i = 0; i < n; ++i) {
    auto it = clients_.find(ids[i]);
    if (it == clients_.end()) throw std::out_of_range("unknown client id " + std::to_string(ids[i]));
    host_ptrs_[i] = it->second.bv.p;
    host_ptrs_[n + i] = it->second.gsw.p;
  }
  grow_ptr_slots(2ull * n);
  PtrSlot &sl = ring_[ring_next_++ % kPtrSlots];
  ck(cudaEventSynchronize(sl.done), "key pointer slot");
  std::copy(host_ptrs_.begin(), host_ptrs_.end(), sl.host);
  ck(cudaMemcpyAsync(keyptrs_.p, sl.host, 2ull * n * sizeof(void *), cudaMemcpyHostToDevice, st_),
     "key pointers");
  ck(cudaEventRecord(sl.done, st_), "event record");
}

// ------------------------------------------------------------------ pipeline
void Server::stage_in(const uint64_t *d_queries, uint32_t n) {
  ck(cudaMemcpy2DAsync(lvl_[0].p, lvl_slots_ * ct_ * 8, d_queries, ct_ * 8, ct_ * 8, n,
                       cudaMemcpyDeviceToDevice, st_), "query staging");
}

// When ntt_first is given and the batch and layout allow it (two or more
// queries, an even first dimension under at least one expansion level;
// OPIR_NTT_LEAVES=0 turns it off), the last level writes the first n0
// leaves in NTT form and *ntt_first is set.
const uint64_t *Server::run_expand(uint32_t n, bool *ntt_first) {
  const uint64_t level_stride = static_cast<uint64_t>(kLKsRows) * row_;
  const char *env = std::getenv("OPIR_NTT_LEAVES");
  // a single query keeps the coefficient path: its last level is too
  // small for the NTT-form tail to pay for itself (CONFIG_N2048_K1 batch 1:
  // 561 vs 550 q/s)
  const bool ntt = ntt_first && n >= 2 && !(env && env[0] == '0') && sh_.h >= 1 &&
                   sh_.n0 % 2 == 0 && sh_.n0 / 2 <= expand_nodes(sh_, sh_.h - 1);
  for (uint32_t d = 0; d < sh_.h; ++d)
    if (k1_)
      opir1::launch_expand_level(d1(), sh_, d, lvl_[d & 1].p, lvl_slots_, lvl_[(d + 1) & 1].p,
                                 lvl_slots_, keyptrs_.p, level_stride, n, st_,
                                 ntt && d + 1 == sh_.h ? sh_.n0 / 2 : 0);
    else
      launch_expand_level(dp_, sh_, d, lvl_[d & 1].p, lvl_slots_, lvl_[(d + 1) & 1].p, lvl_slots_,
                          keyptrs_.p, level_stride, n, st_,
                          ntt && d + 1 == sh_.h ? sh_.n0 / 2 : 0);
  if (ntt_first) *ntt_first = ntt;
  return lvl_[sh_.h & 1].p;
}

// Tensor-core scan of n queries: 16 columns per tile up to 8 queries, else
// 32 (column tiles of one row tile run on neighbouring CTAs, so the
// database tile is read from HBM once).
void Server::launch_scan(const uint8_t *qb, uint64_t *cmat, uint32_t n) {
  const uint32_t ncols = 2 * n;
  Tc4Args a{};
  a.ntile = ncols <= 16 ? 16 : 32;
  a.stages = scan_tc4_max_stages(a.ntile);
  a.k_tiles = (sh_.n0p + 63) / 64;
  a.other = sh_.other;
  a.m_tiles = (sh_.other + 127) / 128;
  a.ncols = ncols;
  a.col_tiles = (ncols + a.ntile - 1) / a.ntile;
  a.zcount = n_ * limbs_;
  a.cmat = cmat;
  a.err = err_.p;
  a.progress = progress_.p;
  a.wait_cycles = scan_wait_;
  CUtensorMap map_q;
  opir::make_plane_map(&map_q, qb, sh_.n0p, ncols, static_cast<uint64_t>(n_) * limbs_ * 8, a.ntile,
                       64);
  launch_scan_tc4(map_db_, map_q, a, sm_count_, st_);
}

// Reads and clears the tensor-core scan's error word (stream must be idle).
void Server::check_device_error() {
  uint32_t e = 0;
  ck(cudaMemcpy(&e, err_.p, sizeof(e), cudaMemcpyDeviceToHost), "error word");
  if (e != 0) {
    ck(cudaMemset(err_.p, 0, sizeof(e)), "error word");
    throw std::runtime_error("tensor-core scan timed out (code " + std::to_string(e) + ")");
  }
}

// First dimension: NTT of the first n0 leaves into the query matrix (in the
// expansion buffer that does not hold the leaves), its byte planes (in the
// leaves' buffer, dead by then), the scan (its output back in the first
// buffer), INTT into mid_[0].
// Records stage mark i of a timed call; inside a capture it becomes an
// event-record node that later calls retarget to their own events.
void Server::mark(Events ev, int i) {
  if (!ev) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ck(cudaStreamIsCapturing(st_, &cs), "capture status");
  if (cs == cudaStreamCaptureStatusActive)
    ck(cudaEventRecordWithFlags(ev[i], st_, cudaEventRecordExternal), "event record");
  else
    ck(cudaEventRecord(ev[i], st_), "event record");
}

void Server::run_first_dim(const uint64_t *leaves, uint32_t n, Events ev, bool leaves_ntt) {
  const int li = leaves == lvl_[0].p ? 0 : 1;
  uint64_t *qm = lvl_[li ^ 1].p;
  uint8_t *qb = reinterpret_cast<uint8_t *>(lvl_[li].p);
  uint64_t *cmat = lvl_[li ^ 1].p;
  if (leaves_ntt) {
    // NTT-form leaves: byte planes into the other buffer (the last
    // expansion level's input, dead now), the scan's output over the leaves
    qb = reinterpret_cast<uint8_t *>(lvl_[li ^ 1].p);
    cmat = lvl_[li].p;
    if (k1_) opir1::launch_fst_pack_leaves(sh_, leaves, lvl_slots_, qb, n, st_);
    else launch_fst_pack_leaves(sh_, leaves, lvl_slots_, qb, n, st_);
  } else if (k1_) {
    opir1::launch_fst_ntt(d1(), sh_, leaves, lvl_slots_, qm, n, st_);
    opir1::launch_fst_pack(sh_, qm, qb, n, st_);
  } else {
    launch_fst_ntt(dp_, sh_, leaves, lvl_slots_, qm, n, st_);
    launch_fst_pack(sh_, qm, qb, n, st_);
  }
  mark(ev, 6);
  launch_scan(qb, cmat, n);
  mark(ev, 7);
  if (k1_) opir1::launch_epilogue(d1(), sh_, cmat, mid_[0].p, sh_.other, n, st_);
  else launch_epilogue(dp_, sh_, cmat, mid_[0].p, sh_.other, n, st_);
}

const uint64_t *Server::run_other_dims(uint32_t n) {
  const uint32_t levels = tree_h_;
  for (uint32_t a = 0; a < levels; ++a)
    run_mux(sh_, a, levels, mid_[a & 1].p, mid_[(a + 1) & 1].p, sh_.other, sel_.p, n);
  return mid_[levels & 1].p;
}

// The kernels of one batch, queries d_queries -> responses d_resp (key
// pointers already uploaded).
void Server::enqueue_core(uint32_t n, const uint64_t *d_queries, uint64_t *d_resp, Events ev) {
  mark(ev, 0);
  stage_in(d_queries, n);
  bool leaves_ntt = false;
  const uint64_t *leaves = run_expand(n, &leaves_ntt);
  mark(ev, 1);
  run_selectors(leaves, keyptrs_.p + n, n);
  mark(ev, 2);
  run_first_dim(leaves, n, ev, leaves_ntt);
  mark(ev, 3);
  const uint64_t *res = run_other_dims(n);
  mark(ev, 4);
  if (shard_)  // row shard: the partial ciphertext, before the last levels
    ck(cudaMemcpy2DAsync(d_resp, ct_ * 8, res, static_cast<size_t>(sh_.other) * ct_ * 8, ct_ * 8, n,
                         cudaMemcpyDeviceToDevice, st_), "partial copy");
  else
    run_modswitch(res, sh_.other, d_resp, n);
  mark(ev, 5);
}

// Replays (capturing on the second use) the pipeline of a batch of n from
// the staging buffer q_in_ to resp_.
void Server::launch_graph(uint32_t n, Events ev) {
  const auto key = std::make_tuple(n, ev != nullptr);
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    if (!graph_seen_.count(key)) {  // first use: eager (warms one-time setup)
      graph_seen_.insert(key);
      enqueue_core(n, q_in_.p, resp_.p, ev);
      return;
    }
    const uint64_t l0 = launch_count();
    Graph g;
    ck(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      enqueue_core(n, q_in_.p, resp_.p, ev);
    } catch (...) {
      cudaGraph_t partial = nullptr;
      cudaStreamEndCapture(st_, &partial);
      if (partial) cudaGraphDestroy(partial);
      cudaGetLastError();
      throw;
    }
    ck(cudaStreamEndCapture(st_, &g.graph), "end capture");
    g.kernels = launch_count() - l0;
    note_launches(-static_cast<int64_t>(g.kernels));  // counted on replay
    if (ev) {
      size_t count = 0;
      ck(cudaGraphGetNodes(g.graph, nullptr, &count), "graph nodes");
      std::vector<cudaGraphNode_t> nodes(count);
      ck(cudaGraphGetNodes(g.graph, nodes.data(), &count), "graph nodes");
      g.ev_nodes.assign(kMarks, nullptr);
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        ck(cudaGraphNodeGetType(nd, &ty), "node type");
        if (ty != cudaGraphNodeTypeEventRecord) continue;
        cudaEvent_t e = nullptr;
        ck(cudaGraphEventRecordNodeGetEvent(nd, &e), "node event");
        for (int i = 0; i < kMarks; ++i)
          if (ev[i] == e) g.ev_nodes[i] = nd;
      }
    }
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, g.graph, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g.graph);
      ck(ie, "graph instantiate");
    }
    it = graphs_.emplace(key, g).first;
  }
  if (ev)
    for (int i = 0; i < kMarks; ++i)
      if (it->second.ev_nodes[i])
        ck(cudaGraphExecEventRecordNodeSetEvent(it->second.exec, it->second.ev_nodes[i], ev[i]),
           "event node");
  ck(cudaGraphLaunch(it->second.exec, st_), "graph launch");
  note_launches(static_cast<int64_t>(it->second.kernels));
}

void Server::run_pipeline(uint32_t n, const uint64_t *ids, const uint64_t *d_queries,
                          uint64_t *d_resp, Events ev) {
  if (!db_loaded_) throw std::runtime_error("make_query before load_data");
  if (n == 0) return;
  ensure_capacity(n);
  upload_keyptrs(ids, n);
  if (!use_graphs_) {
    enqueue_core(n, d_queries, d_resp, ev);
    return;
  }
  if (d_queries != q_in_.p)
    ck(cudaMemcpyAsync(q_in_.p, d_queries, static_cast<size_t>(n) * ct_ * 8,
                       cudaMemcpyDeviceToDevice, st_), "query staging");
  launch_graph(n, ev);
  if (d_resp != resp_.p)
    ck(cudaMemcpyAsync(d_resp, resp_.p, static_cast<size_t>(n) * out_words_ * 8,
                       cudaMemcpyDeviceToDevice, st_), "response copy");
}

void Server::make_query_batch(uint32_t n, const uint64_t *ids, const uint64_t *queries,
                              uint64_t *responses, Events ev) {
  check_ct_values(queries, n);
  if (!db_loaded_) throw std::runtime_error("make_query before load_data");
  if (n == 0) return;
  ensure_capacity(n);
  ck(cudaMemcpyAsync(q_in_.p, queries, static_cast<size_t>(n) * ct_ * 8, cudaMemcpyHostToDevice,
                     st_), "query upload");
  run_pipeline(n, ids, q_in_.p, resp_.p, ev);
  ck(cudaMemcpyAsync(responses, resp_.p, static_cast<size_t>(n) * out_words_ * 8,
                     cudaMemcpyDeviceToHost, st_), "response download");
  ck(cudaStreamSynchronize(st_), "make_query");
  check_device_error();
}

void Server::combine_device(uint32_t n, const uint64_t *d_partials, uint64_t *d_responses) {
  if (!shard_) throw std::invalid_argument("combine_shards needs a row shard");
  const uint32_t G = num_shards_, h = sh_.num_dims - 1;
  const uint64_t words = static_cast<uint64_t>(n) * G * ct_;
  for (auto &b : comb_)
    if (b.n < words) b.alloc(words);
  for (uint32_t g = 0; g < G; ++g)  // query i's G ciphertexts side by side
    ck(cudaMemcpy2DAsync(comb_[0].p + static_cast<uint64_t>(g) * ct_, static_cast<size_t>(G) * ct_ * 8,
                         d_partials + static_cast<uint64_t>(g) * n * ct_, ct_ * 8, ct_ * 8, n,
                         cudaMemcpyDeviceToDevice, st_), "partial gather");
  int cur = 0;
  for (uint32_t a = tree_h_; a < h; ++a, cur ^= 1)
    run_mux(sh_, a, h, comb_[cur].p, comb_[cur ^ 1].p, G, sel_.p, n);
  run_modswitch(comb_[cur].p, G, d_responses, n);
}

void Server::combine_host(uint32_t n, const uint64_t *partials, uint64_t *responses) {
  const size_t cts = static_cast<size_t>(num_shards_) * n;
  check_ct_values(partials, cts);
  opir::DevBuf<uint64_t> d_in, d_out;
  d_in.alloc(cts * ct_);
  d_out.alloc(static_cast<size_t>(n) * 2 * kN);
  ck(cudaMemcpyAsync(d_in.p, partials, cts * ct_ * 8, cudaMemcpyHostToDevice, st_), "upload");
  combine_device(n, d_in.p, d_out.p);
  ck(cudaMemcpyAsync(responses, d_out.p, static_cast<size_t>(n) * 2 * kN * 8,
                     cudaMemcpyDeviceToHost, st_), "download");
  ck(cudaStreamSynchronize(st_), "combine_shards");
  check_device_error();
}

void Server::make_query_batch_device(uint32_t n, const uint64_t *ids, const uint64_t *d_queries,
                                     uint64_t *d_responses, Events ev) {
  run_pipeline(n, ids, d_queries, d_responses, ev);
}

// ------------------------------------------------------------------ stages
void Server::expand_query(uint64_t id, const uint64_t *query, uint64_t *out) {
  check_ct_values(query, 1);
  ensure_capacity(1);
  upload_keyptrs(&id, 1);
  ck(cudaMemcpyAsync(lvl_[0].p, query, ct_ * 8, cudaMemcpyHostToDevice, st_), "upload");
  const uint64_t *leaves = run_expand(1);
  ck(cudaMemcpyAsync(out, leaves, static_cast<size_t>(sh_.useful) * ct_ * 8,
                     cudaMemcpyDeviceToHost, st_), "download");
  ck(cudaStreamSynchronize(st_), "expand_query");
}

void Server::complete_selectors(uint64_t id, const uint64_t *expanded, uint64_t *out) {
  check_ct_values(expanded, sh_.useful);
  ensure_capacity(1);
  upload_keyptrs(&id, 1);
  const uint32_t nsel = sh_.num_dims - 1;
  if (nsel == 0) {
    ck(cudaStreamSynchronize(st_), "complete_selectors");
    return;
  }
  ck(cudaMemcpyAsync(lvl_[0].p, expanded, static_cast<size_t>(sh_.useful) * ct_ * 8,
                     cudaMemcpyHostToDevice, st_), "upload");
  run_selectors(lvl_[0].p, keyptrs_.p + 1, 1);
  // the rows without their Shoup companions
  ck(cudaMemcpy2DAsync(out, ct_ * 8, sel_.p, row_ * 8, ct_ * 8,
                       static_cast<size_t>(nsel) * 2 * sh_.l_ep, cudaMemcpyDeviceToHost, st_),
     "download");
  ck(cudaStreamSynchronize(st_), "complete_selectors");
}

void Server::evaluate_first_dim(const uint64_t *fst_query, uint64_t *out) {
  if (!db_loaded_) throw std::runtime_error("evaluate_first_dim before load_data");
  check_ct_values(fst_query, sh_.n0);
  ensure_capacity(1);
  ck(cudaMemcpyAsync(lvl_[0].p, fst_query, static_cast<size_t>(sh_.n0) * ct_ * 8,
                     cudaMemcpyHostToDevice, st_), "upload");
  run_first_dim(lvl_[0].p, 1, nullptr);
  ck(cudaMemcpyAsync(out, mid_[0].p, static_cast<size_t>(sh_.other) * ct_ * 8,
                     cudaMemcpyDeviceToHost, st_), "download");
  ck(cudaStreamSynchronize(st_), "evaluate_first_dim");
  check_device_error();
}

void Server::evaluate_other_dim(const uint64_t *mid, const uint64_t *selectors, uint64_t *out) {
  const uint32_t nsel = sh_.num_dims - 1;
  if (nsel && sh_.other < (1u << (nsel - 1)))
    throw std::invalid_argument("evaluate_other_dim: layout has fewer candidates than its selector tree");
  check_ct_values(mid, sh_.other);
  if (nsel) check_ct_values(selectors, static_cast<size_t>(nsel) * 2 * sh_.l_ep);
  ensure_capacity(1);
  ck(cudaMemcpyAsync(mid_[0].p, mid, static_cast<size_t>(sh_.other) * ct_ * 8,
                     cudaMemcpyHostToDevice, st_), "upload");
  std::vector<uint64_t> rows;
  if (nsel) {
    const size_t n_rows = static_cast<size_t>(nsel) * 2 * sh_.l_ep;
    rows.reserve(n_rows * row_);
    for (size_t r = 0; r < n_rows; ++r) append_row(rows, selectors + r * ct_, n_, limbs_);
    ck(cudaMemcpyAsync(sel_.p, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice, st_),
       "upload");
  }
  const uint64_t *r = run_other_dims(1);
  ck(cudaMemcpyAsync(out, r, ct_ * 8, cudaMemcpyDeviceToHost, st_), "download");
  ck(cudaStreamSynchronize(st_), "evaluate_other_dim");
}

void Server::ext_prod_mux(const uint64_t *x, const uint64_t *y, const uint64_t *sel,
                          uint64_t *out) {
  check_ct_values(x, 1);
  check_ct_values(y, 1);
  const size_t n_rows = 2ull * sh_.l_ep;
  check_ct_values(sel, n_rows);
  Shape4 sh = sh_;  // one MUX level of a two-candidate tree
  sh.other = 2;
  sh.num_dims = 2;
  std::vector<uint64_t> rows;
  rows.reserve(n_rows * row_);
  for (size_t r = 0; r < n_rows; ++r) append_row(rows, sel + r * ct_, n_, limbs_);
  opir::DevBuf<uint64_t> xy, res, srows;
  xy.alloc(2 * ct_);
  res.alloc(2 * ct_);
  srows.alloc(rows.size());
  ck(cudaMemcpyAsync(xy.p, x, ct_ * 8, cudaMemcpyHostToDevice, st_), "upload");
  ck(cudaMemcpyAsync(xy.p + ct_, y, ct_ * 8, cudaMemcpyHostToDevice, st_), "upload");
  ck(cudaMemcpyAsync(srows.p, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice, st_), "upload");
  run_mux(sh, 0, 1, xy.p, res.p, 2, srows.p, 1);
  ck(cudaMemcpyAsync(out, res.p, ct_ * 8, cudaMemcpyDeviceToHost, st_), "download");
  ck(cudaStreamSynchronize(st_), "ext_prod_mux");
}

void Server::tree_unpack(uint64_t id, const uint64_t *query) {
  check_ct_values(query, 1);
  upload_keyptrs(&id, 1);
  ck(cudaMemcpyAsync(lvl_[0].p, query, ct_ * 8, cudaMemcpyHostToDevice, st_), "upload");
  const uint64_t *leaves = run_expand(1);
  if (sh_.num_dims > 1)
    run_selectors(leaves, keyptrs_.p + 1, 1);
}

void Server::tree_select_device(const uint64_t *d_leaves, const uint64_t *d_selectors,
                                uint64_t fold_begin, uint64_t fold_count, uint64_t *d_out) {
  if (!db_loaded_) throw std::runtime_error("select_level before load_data");
  ck(cudaMemcpyAsync(lvl_[0].p, d_leaves, static_cast<size_t>(sh_.n0) * ct_ * 8,
                     cudaMemcpyDeviceToDevice, st_), "alpha copy");
  run_first_dim(lvl_[0].p, 1, nullptr);
  const uint32_t fold = static_cast<uint32_t>(fold_count);
  const size_t sel_words = 2ull * sh_.l_ep * row_;  // one selector with companions
  for (uint32_t a = 1; a <= fold; ++a) {  // MSB-first: step a takes selector begin+count-a
    const uint64_t u = fold_begin + fold_count - a;
    ck(cudaMemcpyAsync(sel_.p + a * sel_words, d_selectors + u * sel_words, sel_words * 8,
                       cudaMemcpyDeviceToDevice, st_), "selector copy");
  }
  for (uint32_t a = 1; a <= fold; ++a)
    run_mux(sh_, a, sh_.num_dims - 1, mid_[(a - 1) & 1].p, mid_[a & 1].p, sh_.other, sel_.p, 1);
  ck(cudaMemcpyAsync(d_out, mid_[fold & 1].p, ct_ * 8, cudaMemcpyDeviceToDevice, st_), "result");
}

void Server::select_fold(const uint64_t *alpha, const uint64_t *fold_sel, uint32_t fold,
                         uint64_t *out) {
  if (!db_loaded_) throw std::runtime_error("select_level before load_data");
  check_ct_values(alpha, sh_.n0);
  if (fold) check_ct_values(fold_sel, static_cast<size_t>(fold) * 2 * sh_.l_ep);
  ensure_capacity(1);
  ck(cudaMemcpyAsync(lvl_[0].p, alpha, static_cast<size_t>(sh_.n0) * ct_ * 8,
                     cudaMemcpyHostToDevice, st_), "upload");
  run_first_dim(lvl_[0].p, 1, nullptr);
  const uint64_t *res = mid_[0].p;
  std::vector<uint64_t> rows;
  if (fold) {
    const size_t n_rows = static_cast<size_t>(fold) * 2 * sh_.l_ep;
    rows.reserve(n_rows * row_);
    for (size_t r = 0; r < n_rows; ++r) append_row(rows, fold_sel + r * ct_, n_, limbs_);
    // slot 0 of the selector set is unused: step a takes slot a
    ck(cudaMemcpyAsync(sel_.p + 2ull * sh_.l_ep * row_, rows.data(), rows.size() * 8,
                       cudaMemcpyHostToDevice, st_), "upload");
    for (uint32_t a = 1; a <= fold; ++a)
      run_mux(sh_, a, sh_.num_dims - 1, mid_[(a - 1) & 1].p, mid_[a & 1].p, sh_.other, sel_.p, 1);
    res = mid_[fold & 1].p;
  }
  ck(cudaMemcpyAsync(out, res, ct_ * 8, cudaMemcpyDeviceToHost, st_), "download");
  ck(cudaStreamSynchronize(st_), "select_level");
  check_device_error();
}

}  // namespace opir4
