// C-ABI implementation: the server handle that replaces PirServer's query
// path (src/server.cpp). Host code orchestrates the sm_100a kernels of
// opir_kernels.cu on one CUDA stream per handle; there is no CPU compute
// path -- every arithmetic step of make_query runs in a kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <iterator>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <map>
#include <new>
#include <set>
#include <stdexcept>
#include <tuple>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/onionpir_b200.h"
#include "opir_c4_server.h"
#include "opir_client.h"
#include "opir_host.h"
#include "opir_kernels.h"
#include "opir_params.h"
#include "opir_scan_tc.h"
#include "opir_shard.h"
#include "opir_tree.h"

namespace {

using opir::CudaError;
using opir::ck;
using opir::DevBuf;
using opir::DeviceGuard;

struct ClientKeys {
  DevBuf<uint32_t> bv;   // h x L_KS x 2 polys x 2 residues x N
  DevBuf<uint32_t> gsw;  // 2 L_KEY x 2 polys x 2 residues x N
};

constexpr int kStages = 5;
constexpr int kEvents = kStages + 3;   // 6 stage boundaries + scan begin/end
constexpr int kTimingSlots = 512;

// Pinned staging slot for one call's key-pointer table, so that its upload is
// an asynchronous copy; `done` marks when the copy that read it has run.
struct KeyPtrSlot {
  const uint32_t **host = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
};
constexpr int kKeyPtrSlots = 4;

// Tiling of the tensor-core scan for one batch-size bucket (batches of
// 2^(b-1) < n <= 2^b queries; the last bucket takes every larger batch).
struct ScanTile {
  uint32_t ntile = 0, kt = 0, stages = 0;  // ntile 0: pick by the default rule
};
constexpr int kTileBuckets = 10;

// One captured make_query pipeline: batch size, the scan tiling it was
// captured with and whether it records the stage events; `kernels` =
// launches it replays; ev_nodes[i] = the event-record node of stage mark i.
using GraphKey = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, bool, bool>;
struct GraphEntry {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t kernels = 0;
  std::vector<cudaGraphNode_t> ev_nodes;
};
int tile_bucket(uint32_t n) {
  int b = 0;
  while (b + 1 < kTileBuckets && (1u << b) < n) ++b;
  return b;
}

// Cluster widths of the expansion and MUX levels for one batch bucket
// (opir_server_autotune); 0 = the launchers' default rule.
struct LevelSplits {
  uint8_t exp[16] = {};
  uint8_t mux[32] = {};
};

// OPIR_SPLIT=0 turns every cluster split off (tuned widths included).
bool splits_allowed() {
  const char *e = std::getenv("OPIR_SPLIT");
  return !(e && std::strcmp(e, "0") == 0);
}

}  // namespace

struct opir_server {
  opir_params params{};
  opir::Shape shape{};
  opir::DevParams dp{};
  int device = 0;
  cudaStream_t stream = nullptr;
  DevBuf<uint32_t> tables;
  DevBuf<uint8_t> db8;       // byte-plane database, see opir_kernels.h
  bool db_loaded = false;
  CUtensorMap map_db[2]{};   // TMA views of db8 for the tensor-core scan: 128 B / 64 B swizzle
  ScanTile tile[kTileBuckets];  // tensor-core scan tiling per batch bucket (autotuned)
  LevelSplits split[kTileBuckets];  // level cluster widths per batch bucket (autotuned)
  int sm_count = 148;
  int scan_mode = 0;         // 0 auto, 1 tensor cores, 2 CUDA cores
  DevBuf<uint32_t> err;      // device error word of the tensor-core scan
  long long scan_wait = 0;   // scan pipeline wait limit in cycles (0: default)
  std::unordered_map<uint64_t, ClientKeys> clients;
  std::string last_error;
  // scratch arena (sized for `cap` queries)
  uint32_t cap = 0;
  uint64_t lvl_slots = 1;   // ciphertext slots per query in an expansion buffer
  DevBuf<uint64_t> q_u64, resp_u64;
  DevBuf<uint8_t> resp_bytes;
  DevBuf<uint32_t> lvl[2], sel, cmat, mid[2];
  DevBuf<uint8_t> qb;        // byte-plane first-dimension query matrix
  DevBuf<const uint32_t *> keyptrs;
  std::vector<const uint32_t *> host_keyptrs;
  KeyPtrSlot kp_ring[kKeyPtrSlots];
  uint32_t kp_next = 0;
  // stage timing: one event set per timed call, averaged on request
  bool timing = false;
  std::vector<std::vector<cudaEvent_t>> ev_pool;
  uint32_t timed_calls = 0;
  cudaEvent_t *cur_ev = nullptr;
  // CONFIG_N4096_K2_MP handles forward every call to this object
  std::unique_ptr<opir4::Server> c4;
  // tree level handles (view OPIR_VIEW_MATRIX): the plan's beta fold
  uint64_t tree_b = 0, fold_begin = 0, fold_count = 0;
  // MUX levels answered by make_query: num_dims - 1, or h - log2 G on a row
  // shard (view OPIR_VIEW_ROW_SHARD, opir_shard.h), whose rows are
  // row_map's database rows and whose last batch's client ids are
  // shard_ids (their selectors stay in `sel` for opir_server_combine_shards)
  uint32_t tree_h = 0;
  uint32_t shard = 0, num_shards = 1;
  std::vector<uint32_t> host_rows;
  DevBuf<uint32_t> row_map;
  std::vector<uint64_t> shard_ids;
  DevBuf<uint32_t> comb[2];  // combine: n x num_shards ciphertext slots
  // captured pipelines (see run_pipeline); a key is captured on its second use
  bool use_graphs = true;
  std::map<GraphKey, GraphEntry> graphs;
  std::set<GraphKey> graph_seen;
};

// A whole device-resident tree (see opir_tree_create): the query-shape
// handle, one level handle per level, a join stream and the output buffer.
struct opir_tree {
  opir_tree_params tree{};
  int device = 0;
  opir_server *q = nullptr;
  std::vector<opir_server *> levels;
  cudaStream_t stream = nullptr;
  DevBuf<uint64_t> out;            // (L + 1) x 2N u64
  cudaEvent_t q_done = nullptr;
  std::vector<cudaEvent_t> done;   // per level
  std::string last_error;
};

namespace {

using opir::kCtWords;
using opir::kN;

opir_status fail(std::string *sink, opir_status code, const std::string &msg) {
  if (sink) *sink = msg;
  return code;
}

// Runs f, mapping the exception types the reference throws onto status codes
// and keeping the message in *sink.
template <typename F>
opir_status guarded_to(std::string *sink, F &&f) {
  try {
    f();
    if (sink) sink->clear();
    return OPIR_OK;
  } catch (const std::invalid_argument &e) {
    return fail(sink, OPIR_ERR_INVALID_ARGUMENT, e.what());
  } catch (const std::out_of_range &e) {
    return fail(sink, OPIR_ERR_OUT_OF_RANGE, e.what());
  } catch (const std::overflow_error &e) {
    return fail(sink, OPIR_ERR_OVERFLOW, e.what());
  } catch (const std::bad_alloc &) {
    return fail(sink, OPIR_ERR_NO_MEMORY, "device or host allocation failed");
  } catch (const CudaError &e) {
    cudaGetLastError();
    return fail(sink, OPIR_ERR_CUDA, e.what());
  } catch (const std::runtime_error &e) {
    cudaGetLastError();
    return fail(sink, OPIR_ERR_RUNTIME, e.what());
  } catch (...) {
    return fail(sink, OPIR_ERR_RUNTIME, "unknown error");
  }
}

template <typename F>
opir_status guarded(opir_server *s, F &&f) {
  return guarded_to(s ? &s->last_error : nullptr, std::forward<F>(f));
}

uint32_t resp_bytes_of(const opir_params &p) {
  return static_cast<uint32_t>((2ull * p.poly_degree * p.small_q_width + 7) / 8);
}

// CONFIG_N2048_K2_MP: two 29-bit RNS limbs at N = 2048, the residue pair of
// CONFIG_N2048_K1_COMP with the MP gadgets; runs on the same kernels.
bool is_k2mp(const opir_params &p) { return p.num_limbs == 2 && p.poly_degree == 2048; }

// u64 words of one polynomial at the boundary (queries, keys, stage
// outputs): N values mod q1 q2, or N per RNS limb (limb-major).
uint64_t poly_words(const opir_params &p) {
  return static_cast<uint64_t>(opir::kN) * (is_k2mp(p) ? 2 : 1);
}

// Kernel-facing shape of a layout; *lvl_slots receives the ciphertext slots
// per query that an expansion buffer needs (the widest tree level, at least
// the useful leaves).
opir::Shape make_shape(const opir_params &p, uint64_t *lvl_slots) {
  opir::Shape sh{};
  sh.n0 = static_cast<uint32_t>(p.fst_dim_sz);
  sh.other = static_cast<uint32_t>(p.other_dim_sz);
  sh.num_dims = p.num_dims;
  sh.h = p.expansion_height;
  sh.useful = static_cast<uint32_t>(p.fst_dim_sz + static_cast<uint64_t>(p.l_ep) * (p.num_dims - 1));
  sh.l_ep = p.l_ep;
  sh.l_key = p.l_key;
  sh.l_ks = p.l_ks;
  sh.base_ep = p.base_log2;
  sh.base_key = p.base_log2_key;
  sh.base_ks = p.base_log2_ks;
  sh.num_pt = p.num_pt;
  sh.n0p = static_cast<uint32_t>((p.fst_dim_sz + 15) / 16 * 16);
  sh.gadget = is_k2mp(p) ? 1 : 0;
  uint64_t slots = 1;
  for (uint32_t d2 = 0; d2 < sh.h; ++d2) slots = std::max<uint64_t>(slots, 2ull * opir::expand_nodes(sh, d2));
  *lvl_slots = std::max<uint64_t>(slots, sh.useful);
  return sh;
}

// Element counts of every scratch-arena buffer for n queries; the single
// source for ensure_capacity and opir_plan_memory.
struct ScratchPlan {
  size_t q_u64, resp_u64, resp_bytes, lvl, sel, qb, cmat, mid, keyptrs;
  uint64_t bytes() const {
    return (q_u64 + resp_u64) * 8 + resp_bytes + 2 * lvl * 4 + sel * 4 + qb + cmat * 4 +
           2 * mid * 4 + keyptrs * sizeof(void *);
  }
};

ScratchPlan plan_scratch(const opir::Shape &sh, uint64_t lvl_slots, uint32_t resp_bytes, uint32_t n,
                         uint64_t pw = opir::kN) {
  const uint64_t ct = kCtWords;
  const uint64_t nsel = sh.num_dims > 1 ? sh.num_dims - 1 : 0;
  ScratchPlan pl{};
  pl.q_u64 = static_cast<size_t>(n) * 2 * pw;  // queries at the boundary
  pl.resp_u64 = static_cast<size_t>(n) * 2 * kN;
  pl.resp_bytes = static_cast<size_t>(n) * resp_bytes;
  pl.lvl = n * lvl_slots * ct;
  pl.sel = std::max<uint64_t>(1, n * nsel * 2 * sh.l_ep * ct);
  pl.qb = 2ull * kN * 4 * 2 * n * sh.n0p;
  pl.cmat = 2ull * kN * sh.other * 2 * n;
  pl.mid = static_cast<size_t>(n) * sh.other * ct;
  pl.keyptrs = 2ull * n;
  return pl;
}

void setup_device_params(opir_server *s) {
  const opir_params &p = s->params;
  const auto t1 = opir::make_limb_tables(kN, static_cast<uint32_t>(p.q1), static_cast<uint32_t>(p.w1));
  const auto t2 = opir::make_limb_tables(kN, static_cast<uint32_t>(p.q2), static_cast<uint32_t>(p.w2));
  // per residue: fw, fw_sh, iw, iw_sh (kN each), then (fw, fw_sh) and
  // (iw, iw_sh) interleaved (2 kN each), then (psi^m, Shoup) for m < 2N
  // (4 kN)
  constexpr int kResWords = 12 * kN;
  std::vector<uint32_t> host(2 * kResWords);
  const opir::LimbTables *ts[2] = {&t1, &t2};
  for (int r = 0; r < 2; ++r) {
    uint32_t *h = host.data() + r * kResWords;
    {
      // psi = fw[brev(1)] = fw[N / 2] (fw[k] = psi^brev(k))
      const uint64_t q = ts[r]->q, psi = ts[r]->fw[kN / 2];
      uint64_t pw = 1;
      for (int m = 0; m < 2 * kN; ++m) {
        h[8 * kN + 2 * m] = static_cast<uint32_t>(pw);
        h[8 * kN + 2 * m + 1] = static_cast<uint32_t>((pw << 32) / q);
        pw = pw * psi % q;
      }
      if (pw != 1 || h[8 * kN + 2 * kN] != q - 1)
        throw std::runtime_error("psi is not a primitive 2N-th root of unity");
    }
    std::copy(ts[r]->fw.begin(), ts[r]->fw.end(), h + 0 * kN);
    std::copy(ts[r]->fw_sh.begin(), ts[r]->fw_sh.end(), h + 1 * kN);
    std::copy(ts[r]->iw.begin(), ts[r]->iw.end(), h + 2 * kN);
    std::copy(ts[r]->iw_sh.begin(), ts[r]->iw_sh.end(), h + 3 * kN);
    for (int i = 0; i < kN; ++i) {
      h[4 * kN + 2 * i] = ts[r]->fw[i];
      h[4 * kN + 2 * i + 1] = ts[r]->fw_sh[i];
      h[6 * kN + 2 * i] = ts[r]->iw[i];
      h[6 * kN + 2 * i + 1] = ts[r]->iw_sh[i];
    }
  }
  s->tables.alloc(host.size());
  ck(cudaMemcpy(s->tables.p, host.data(), host.size() * 4, cudaMemcpyHostToDevice), "tables");
  opir::DevParams &d = s->dp;
  for (int r = 0; r < 2; ++r) {
    uint32_t *base = s->tables.p + r * kResWords;
    d.r[r].fw = base + 0 * kN;
    d.r[r].fw_sh = base + 1 * kN;
    d.r[r].iw = base + 2 * kN;
    d.r[r].iw_sh = base + 3 * kN;
    d.r[r].fwt = reinterpret_cast<const uint2 *>(base + 4 * kN);
    d.r[r].iwt = reinterpret_cast<const uint2 *>(base + 6 * kN);
    d.r[r].pwt = reinterpret_cast<const uint2 *>(base + 8 * kN);
    d.r[r].q = ts[r]->q;
    d.r[r].n_inv = ts[r]->n_inv;
    d.r[r].n_inv_sh = ts[r]->n_inv_sh;
    const uint32_t w1n = static_cast<uint32_t>(static_cast<uint64_t>(ts[r]->iw[1]) * ts[r]->n_inv % ts[r]->q);
    d.r[r].w1_ninv = w1n;
    d.r[r].w1_ninv_sh = static_cast<uint32_t>((static_cast<uint64_t>(w1n) << 32) / ts[r]->q);
    d.r[r].mu = ts[r]->mu;
  }
  {
    const uint32_t qs[2] = {ts[0]->q, ts[1]->q};
    const uint32_t *fw[2] = {ts[0]->fw.data(), ts[1]->fw.data()};
    const uint32_t *fw_sh[2] = {ts[0]->fw_sh.data(), ts[1]->fw_sh.data()};
    const uint32_t *iw[2] = {ts[0]->iw.data(), ts[1]->iw.data()};
    const uint32_t *iw_sh[2] = {ts[0]->iw_sh.data(), ts[1]->iw_sh.data()};
    uint32_t nscale[2][4];
    for (int r = 0; r < 2; ++r) {
      nscale[r][0] = d.r[r].n_inv;
      nscale[r][1] = d.r[r].n_inv_sh;
      nscale[r][2] = d.r[r].w1_ninv;
      nscale[r][3] = d.r[r].w1_ninv_sh;
    }
    opir::upload_ntt_constants(qs, fw, fw_sh, iw, iw_sh, nscale);
  }
  d.q = p.q;
  d.half_q = p.q >> 1;
  d.q1 = static_cast<uint32_t>(p.q1);
  d.q2 = static_cast<uint32_t>(p.q2);
  d.q1_inv = static_cast<uint32_t>(p.q1_inv_mod_q2);
  d.q1_inv_sh = static_cast<uint32_t>((static_cast<uint64_t>(d.q1_inv) << 32) / d.q2);
  d.small_q = p.small_q;
  d.small_q_width = p.small_q_width;
  d.limbs = is_k2mp(p) ? 2 : 1;

  s->shape = make_shape(p, &s->lvl_slots);
}

// Drops every captured pipeline (their buffer pointers or tilings changed).
void clear_graphs(opir_server *s) {
  for (auto &kv : s->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  s->graphs.clear();
  s->graph_seen.clear();
}

void ensure_capacity(opir_server *s, uint32_t n) {
  if (n <= s->cap) return;
  clear_graphs(s);
  const ScratchPlan pl =
      plan_scratch(s->shape, s->lvl_slots, resp_bytes_of(s->params), n, poly_words(s->params));
  s->q_u64.alloc(pl.q_u64);
  s->resp_u64.alloc(pl.resp_u64);
  s->resp_bytes.alloc(pl.resp_bytes);
  for (auto &b : s->lvl) b.alloc(pl.lvl);
  s->sel.alloc(pl.sel);
  s->qb.alloc(pl.qb);
  s->cmat.alloc(pl.cmat);
  for (auto &b : s->mid) b.alloc(pl.mid);
  s->keyptrs.alloc(pl.keyptrs);
  s->cap = n;
}

const ClientKeys &client(const opir_server *s, uint64_t id) {
  auto it = s->clients.find(id);
  if (it == s->clients.end()) throw std::out_of_range("unknown client id " + std::to_string(id));
  return it->second;
}

// Makes every pinned key-pointer slot hold at least `entries` pointers.
void grow_keyptr_slots(opir_server *s, size_t entries) {
  for (KeyPtrSlot &sl : s->kp_ring) {
    if (!sl.done) ck(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "event");
    if (sl.cap >= entries) continue;
    ck(cudaEventSynchronize(sl.done), "key pointer slot");
    if (sl.host) cudaFreeHost(sl.host);
    sl.host = nullptr;
    sl.cap = 0;
    ck(cudaMallocHost(reinterpret_cast<void **>(&sl.host), entries * sizeof(void *)), "cudaMallocHost");
    sl.cap = entries;
  }
}

// Uploads the per-query key pointer table (bv pointers then gsw pointers)
// from a pinned slot of a small ring; a slot is refilled only after the copy
// that last read it has executed, which in steady state has long happened.
void upload_keyptrs(opir_server *s, const uint64_t *client_ids, uint32_t n) {
  s->host_keyptrs.resize(2ull * n);
  for (uint32_t i = 0; i < n; ++i) {
    const ClientKeys &k = client(s, client_ids[i]);
    s->host_keyptrs[i] = k.bv.p;
    s->host_keyptrs[n + i] = k.gsw.p;
  }
  grow_keyptr_slots(s, 2ull * n);
  KeyPtrSlot &sl = s->kp_ring[s->kp_next++ % kKeyPtrSlots];
  ck(cudaEventSynchronize(sl.done), "key pointer slot");
  std::copy(s->host_keyptrs.begin(), s->host_keyptrs.end(), sl.host);
  ck(cudaMemcpyAsync(s->keyptrs.p, sl.host, 2ull * n * sizeof(void *), cudaMemcpyHostToDevice,
                     s->stream), "key pointers");
  ck(cudaEventRecord(sl.done, s->stream), "event record");
}

void begin_timed_call(opir_server *s) {
  s->cur_ev = nullptr;
  if (!s->timing || s->timed_calls >= kTimingSlots) return;
  if (s->ev_pool.size() <= s->timed_calls) {
    std::vector<cudaEvent_t> evs(kEvents);
    for (auto &e : evs) ck(cudaEventCreate(&e), "cudaEventCreate");
    s->ev_pool.push_back(std::move(evs));
  }
  s->cur_ev = s->ev_pool[s->timed_calls++].data();
}

void mark(opir_server *s, int i) {
  if (!s->cur_ev) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  ck(cudaStreamIsCapturing(s->stream, &cs), "capture status");
  if (cs == cudaStreamCaptureStatusActive)  // becomes an event-record node of the graph
    ck(cudaEventRecordWithFlags(s->cur_ev[i], s->stream, cudaEventRecordExternal),
       "cudaEventRecord");
  else
    ck(cudaEventRecord(s->cur_ev[i], s->stream), "cudaEventRecord");
}

// Event slot of a two-limb call (null when stage timing is off).
cudaEvent_t *c4_events(opir_server *s) {
  begin_timed_call(s);
  cudaEvent_t *ev = s->cur_ev;
  s->cur_ev = nullptr;
  return ev;
}

// CONFIG_N2048_K1: one 60-bit prime at N = 2048 (no composite split).
bool is_k1p(const opir_params &p) {
  return p.num_limbs == 1 && p.poly_degree == 2048 && p.q1 == 0;
}
// Handles whose limbs are 64-bit words forward to opir4::Server:
// CONFIG_N4096_K2_MP and CONFIG_N2048_K1.
bool is_c4(const opir_params &p) {
  return (p.num_limbs == 2 && p.poly_degree == 4096) || is_k1p(p);
}

// Expansion (Algorithm 2) over n queries whose residue pairs sit in slot 0 of
// lvl[0]; returns the buffer holding the leaves.
// The handle's shape with the cluster widths tuned for a batch of n.
opir::Shape level_shape(const opir_server *s, uint32_t n) {
  opir::Shape sh = s->shape;
  if (splits_allowed()) {
    const LevelSplits &ls = s->split[tile_bucket(n)];
    std::copy(std::begin(ls.exp), std::end(ls.exp), sh.split_exp);
    std::copy(std::begin(ls.mux), std::end(ls.mux), sh.split_mux);
  }
  return sh;
}

// OPIR_NTT_LEAVES=0 keeps every leaf in coefficient form (the first
// dimension then runs its own forward NTT of the leaves).
bool ntt_leaves_allowed() {
  const char *e = std::getenv("OPIR_NTT_LEAVES");
  return !(e && e[0] == '0');
}

// When ntt_first is given and the layout allows it (an even first dimension
// under at least one expansion level), the last level writes the first n0
// leaves in NTT form and *ntt_first is set; the other leaves stay in
// coefficient form.
uint32_t *run_expand(opir_server *s, uint32_t n, bool *ntt_first = nullptr) {
  const opir::Shape sh = level_shape(s, n);
  const uint64_t bv_level_stride = static_cast<uint64_t>(sh.l_ks) * 4 * kN;
  const bool ntt = ntt_first && ntt_leaves_allowed() && sh.h >= 1 && sh.n0 % 2 == 0 &&
                   sh.n0 / 2 <= opir::expand_nodes(sh, sh.h - 1);
  for (uint32_t d = 0; d < sh.h; ++d)
    opir::launch_expand_level(s->dp, sh, d, s->lvl[d & 1].p, s->lvl_slots, s->lvl[(d + 1) & 1].p,
                              s->lvl_slots, s->keyptrs.p, bv_level_stride, n, s->stream,
                              ntt && d + 1 == sh.h ? sh.n0 / 2 : 0);
  if (ntt_first) *ntt_first = ntt;
  return s->lvl[sh.h & 1].p;
}

// Batch sizes from which the tensor-core scan is used in auto mode.
constexpr uint32_t kTcMinBatch = 1;

// Tensor-core scan of n queries with an explicit tiling.
void launch_scan_tc_tile(opir_server *s, uint32_t n, const ScanTile &t) {
  const opir::Shape &sh = s->shape;
  const uint32_t ncols = 2 * n;
  opir::TcScanArgs a{};
  a.ntile = t.ntile;
  a.kt = t.kt;
  a.stages = t.stages;
  a.col_tiles = (ncols + a.ntile - 1) / a.ntile;
  a.k_tiles = (sh.n0p + a.kt - 1) / a.kt;
  a.other = sh.other;
  a.m_tiles = (sh.other + 127) / 128;
  a.ncols = ncols;
  a.zcount = 2 * kN;
  a.levels_per_res = kN;
  for (int r = 0; r < 2; ++r) {
    a.q[r] = s->dp.r[r].q;
    a.mu[r] = s->dp.r[r].mu;
    uint64_t w = 1;
    for (int sft = 0; sft < 7; ++sft) {
      a.w[r][sft] = static_cast<uint32_t>(w);
      w = (w << 8) % a.q[r];
    }
  }
  a.cmat = s->cmat.p;
  a.err = s->err.p;
  a.wait_cycles = s->scan_wait;
  CUtensorMap map_q;
  opir::make_plane_map(&map_q, s->qb.p, sh.n0p, ncols, 2ull * kN * 4, a.ntile, a.kt);
  opir::launch_scan_tc(s->map_db[a.kt == 128 ? 0 : 1], map_q, a, s->sm_count, s->stream);
}

// The tiling a batch of n queries uses: the OPIR_SCAN_TILE override
// ("ntile,kt,stages"), else the autotuned bucket, else the default rule.
ScanTile effective_tile(const opir_server *s, uint32_t n) {
  if (const char *e = std::getenv("OPIR_SCAN_TILE")) {
    unsigned a0 = 0, a1 = 0, a2 = 0;
    if (std::sscanf(e, "%u,%u,%u", &a0, &a1, &a2) == 3) return ScanTile{a0, a1, a2};
  }
  ScanTile t = s->tile[tile_bucket(n)];
  if (t.ntile != 0) return t;
  // ntile <= 32: two accumulator sets of 7 ntile columns ring in TMEM;
  // ntile = 64: one set, a batch of 32 queries in one pass over the database
  const uint32_t ncols = 2 * n;
  t.ntile = ncols <= 16 ? 16 : ncols <= 32 ? 32 : 64;
  t.kt = 128;
  t.stages = opir::scan_tc_max_stages(t.ntile, t.kt);
  return t;
}

void launch_scan_any(opir_server *s, uint32_t n) {
  const opir::Shape &sh = s->shape;
  // the tensor-core form needs n0 <= 8192 (int32 accumulators, see
  // opir_scan_tc.cu); larger first dimensions use the CUDA-core form
  const bool tc_ok = sh.n0p <= 8192;
  const bool tc = tc_ok && (s->scan_mode == 1 || (s->scan_mode == 0 && n >= kTcMinBatch));
  if (!tc) {
    opir::launch_scan(s->dp, sh, s->db8.p, s->qb.p, s->cmat.p, n, s->stream);
    return;
  }
  launch_scan_tc_tile(s, n, effective_tile(s, n));
}

// First dimension: NTT + transpose of the first n0 leaves (the transpose
// alone when the leaves are already in NTT form), scan, gather + INTT.
void run_first_dim(opir_server *s, const uint32_t *leaves, uint32_t n, bool leaves_ntt = false) {
  const opir::Shape &sh = s->shape;
  if (leaves_ntt) {
    opir::launch_fst_pack(sh, leaves, s->lvl_slots, s->qb.p, n, s->stream);
  } else {
    // the NTT-form leaves go to whichever expansion buffer does not hold them
    uint32_t *ntt = leaves == s->lvl[0].p ? s->lvl[1].p : s->lvl[0].p;
    opir::launch_fst_prep(s->dp, sh, leaves, s->lvl_slots, ntt, s->lvl_slots, s->qb.p, n,
                          s->stream);
  }
  mark(s, kStages + 1);
  launch_scan_any(s, n);
  mark(s, kStages + 2);
  opir::launch_scan_epilogue(s->dp, sh, s->cmat.p, s->mid[0].p, sh.other, n, s->stream);
}

// Remaining dimensions: returns the buffer whose slot 0 holds the result.
uint32_t *run_other_dims(opir_server *s, uint32_t n) {
  const opir::Shape sh = level_shape(s, n);
  const uint32_t levels = s->tree_h;
  for (uint32_t a = 0; a < levels; ++a)
    opir::launch_mux_level(s->dp, sh, a, levels, s->mid[a & 1].p, s->mid[(a + 1) & 1].p, sh.other,
                           s->sel.p, n, s->stream);
  return s->mid[levels & 1].p;
}

bool is_row_shard(const opir_server *s) { return s->params.view == OPIR_VIEW_ROW_SHARD; }

// The kernels of one make_query batch, from queries in d_queries to
// responses in d_resp (key pointers already uploaded). Stage marks are
// recorded when a timed call is open.
void enqueue_core(opir_server *s, uint32_t n, const uint64_t *d_queries, uint64_t *d_resp,
                  uint8_t *d_bytes) {
  const opir::Shape &sh = s->shape;
  mark(s, 0);
  opir::launch_split_u64(s->dp, d_queries, s->lvl[0].p, n, 2, s->lvl_slots * kCtWords, s->stream);
  bool leaves_ntt = false;
  const uint32_t *leaves = run_expand(s, n, &leaves_ntt);
  mark(s, 1);
  opir::launch_selectors(s->dp, sh, leaves, s->lvl_slots, s->keyptrs.p + n, s->sel.p, n, s->stream);
  mark(s, 2);
  run_first_dim(s, leaves, n, leaves_ntt);
  mark(s, 3);
  const uint32_t *res = run_other_dims(s, n);
  mark(s, 4);
  if (is_row_shard(s))  // the shard's partial ciphertext, mod q, before the last levels
    opir::launch_compose_u64(s->dp, res, sh.other * kCtWords, d_resp, n, 2, s->stream);
  else
    opir::launch_modswitch(s->dp, res, sh.other, d_resp, d_bytes, resp_bytes_of(s->params), n,
                           s->stream);
  mark(s, 5);
}

// Replays (capturing on the second use) the pipeline of a batch of n from the
// handle's staging buffers q_u64 -> resp_u64. The graph holds fixed buffer
// pointers, so it is dropped whenever the scratch arena grows or the tiling
// changes; the key-pointer upload stays outside it.
void launch_graph(opir_server *s, uint32_t n) {
  const ScanTile t = effective_tile(s, n);
  const bool tc = s->shape.n0p <= 8192 &&
                  (s->scan_mode == 1 || (s->scan_mode == 0 && n >= kTcMinBatch));
  const bool timed = s->cur_ev != nullptr;
  const GraphKey key{n, t.ntile, t.kt, t.stages, tc, timed};
  auto it = s->graphs.find(key);
  if (it == s->graphs.end()) {
    if (!s->graph_seen.count(key)) {  // first use: run eagerly (warms one-time setup)
      s->graph_seen.insert(key);
      enqueue_core(s, n, s->q_u64.p, s->resp_u64.p, nullptr);
      return;
    }
    const uint64_t l0 = opir::launch_count();
    GraphEntry e;
    ck(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
      enqueue_core(s, n, s->q_u64.p, s->resp_u64.p, nullptr);
    } catch (...) {
      cudaGraph_t partial = nullptr;
      cudaStreamEndCapture(s->stream, &partial);
      if (partial) cudaGraphDestroy(partial);
      cudaGetLastError();
      throw;
    }
    ck(cudaStreamEndCapture(s->stream, &e.graph), "end capture");
    e.kernels = opir::launch_count() - l0;
    opir::note_launches(-static_cast<int64_t>(e.kernels));  // counted on replay
    if (timed) {  // find the node of every stage mark, to retarget them per call
      size_t count = 0;
      ck(cudaGraphGetNodes(e.graph, nullptr, &count), "graph nodes");
      std::vector<cudaGraphNode_t> nodes(count);
      ck(cudaGraphGetNodes(e.graph, nodes.data(), &count), "graph nodes");
      e.ev_nodes.assign(kEvents, nullptr);
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        ck(cudaGraphNodeGetType(nd, &ty), "node type");
        if (ty != cudaGraphNodeTypeEventRecord) continue;
        cudaEvent_t ev = nullptr;
        ck(cudaGraphEventRecordNodeGetEvent(nd, &ev), "node event");
        for (int i = 0; i < kEvents; ++i)
          if (s->cur_ev[i] == ev) e.ev_nodes[i] = nd;
      }
    }
    const cudaError_t ie = cudaGraphInstantiate(&e.exec, e.graph, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(e.graph);
      ck(ie, "graph instantiate");
    }
    it = s->graphs.emplace(key, e).first;
  }
  if (timed)  // this call's event slot
    for (int i = 0; i < kEvents; ++i)
      if (it->second.ev_nodes[i])
        ck(cudaGraphExecEventRecordNodeSetEvent(it->second.exec, it->second.ev_nodes[i],
                                                s->cur_ev[i]), "event node");
  ck(cudaGraphLaunch(it->second.exec, s->stream), "graph launch");
  opir::note_launches(static_cast<int64_t>(it->second.kernels));
}

void run_pipeline(opir_server *s, const uint64_t *client_ids, uint32_t n,
                  const uint64_t *d_queries, uint64_t *d_resp, uint8_t *d_bytes) {
  if (!s->db_loaded) throw std::runtime_error("make_query before load_data");
  if (n == 0) return;
  ensure_capacity(s, n);
  upload_keyptrs(s, client_ids, n);
  begin_timed_call(s);
  if (s->use_graphs && d_bytes == nullptr) {
    const size_t qbytes = static_cast<size_t>(n) * 2 * poly_words(s->params) * 8;
    const size_t rbytes = static_cast<size_t>(n) * 2 * kN * 8;
    if (d_queries != s->q_u64.p)
      ck(cudaMemcpyAsync(s->q_u64.p, d_queries, qbytes, cudaMemcpyDeviceToDevice, s->stream),
         "query staging");
    launch_graph(s, n);
    if (d_resp != s->resp_u64.p)
      ck(cudaMemcpyAsync(d_resp, s->resp_u64.p, rbytes, cudaMemcpyDeviceToDevice, s->stream),
         "response copy");
  } else {
    enqueue_core(s, n, d_queries, d_resp, d_bytes);
  }
  s->cur_ev = nullptr;
}

// Reads and clears the tensor-core scan's error word (stream must be idle).
void check_device_error(opir_server *s) {
  uint32_t e = 0;
  ck(cudaMemcpy(&e, s->err.p, sizeof(e), cudaMemcpyDeviceToHost), "error word");
  if (e != 0) {
    ck(cudaMemset(s->err.p, 0, sizeof(e)), "error word");
    throw std::runtime_error("tensor-core scan timed out (code " + std::to_string(e) + ")");
  }
}

void finish(opir_server *s) {
  ck(cudaStreamSynchronize(s->stream), "make_query");
  check_device_error(s);
}

// count: u64 words at the boundary (whole polynomials of poly_words each).
void check_query_values(const opir_server *s, const uint64_t *q, size_t count) {
  if (is_k2mp(s->params)) {  // limb-major: limb (i / N) % 2
    const uint64_t m[2] = {s->params.q1, s->params.q2};
    for (size_t i = 0; i < count; ++i)
      if (q[i] >= m[(i / kN) & 1]) throw std::invalid_argument("query coefficient not reduced mod its limb");
    return;
  }
  for (size_t i = 0; i < count; ++i)
    if (q[i] >= s->params.q) throw std::invalid_argument("query coefficient not reduced mod q");
}

// Database upload in tiles of plaintexts (u16 coefficients). fill(b, e, dst)
// writes database plaintexts [b, e) to dst; on a row shard it is called for
// the shard's plaintexts only, in increasing order.
template <typename Fill>
void load_tiles(opir_server *s, uint64_t logical, Fill &&fill) {
  const opir_params &p = s->params;
  if (logical > p.num_pt)
    throw std::invalid_argument("PirServer::load_data logical plaintext count exceeds its layout");
  const uint64_t local_pt = static_cast<uint64_t>(s->shape.other) * s->shape.n0;
  const uint64_t tile = 16384;
  std::vector<uint16_t> host(tile * kN);
  DevBuf<uint16_t> dev;
  dev.alloc(tile * kN);
  s->db_loaded = false;
  for (uint64_t pb = 0; pb < local_pt; pb += tile) {
    const uint64_t pe = std::min<uint64_t>(local_pt, pb + tile);
    opir::fill_runs(s->host_rows, s->shape.n0, logical, pb, pe, host.data(), fill, kN);
    ck(cudaMemcpyAsync(dev.p, host.data(), (pe - pb) * kN * 2, cudaMemcpyHostToDevice, s->stream),
       "db upload");
    opir::launch_db_preprocess(s->dp, s->shape, dev.p, pb, 0, p.plain_mod, logical, pb, pe,
                               s->row_map.p, s->db8.p, s->stream);
    ck(cudaStreamSynchronize(s->stream), "db preprocess");
  }
  s->db_loaded = true;
}

// The parameters a handle is created on, re-derived from their layout (or
// query shape) so that a caller cannot hand in inconsistent fields.
opir_params checked_params(const opir_params &p) {
  const bool c4 = is_c4(p), k2 = is_k2mp(p);
  if (!c4 && !k2 && (p.poly_degree != static_cast<uint32_t>(kN) || p.num_limbs != 1))
    throw std::invalid_argument(
        "unsupported parameter set (CONFIG_N2048_K1_COMP, CONFIG_N2048_K2_MP or CONFIG_N4096_K2_MP)");
  auto derive = [&](const opir_layout &lay) {
    return is_k1p(p) ? opir::derive_params_k1p(lay)
           : c4     ? opir4::derive(lay)
           : k2     ? opir::derive_params_k2mp(lay)
                    : opir::derive_params(lay);
  };
  if (p.view == OPIR_VIEW_LAYOUT) {
    const opir_params check = derive(opir_layout{p.target_num_pt, p.expansion_height, p.fst_dim_pow2});
    if (check.num_pt != p.num_pt || check.q != p.q || check.q1 != p.q1 || check.q2 != p.q2)
      throw std::invalid_argument("params do not match their layout");
    return check;
  }
  if (p.view == OPIR_VIEW_QUERY_SHAPE) {
    const opir_params scheme = derive(opir_layout{1, 0, 1});
    const opir_params check = opir::with_query_shape(
        scheme, opir_query_shape{p.fst_dim_sz, p.num_dims - 1, p.expansion_height});
    if (check.num_pt != p.num_pt || check.q != p.q || check.q1 != p.q1 || check.q2 != p.q2 ||
        check.num_dims != p.num_dims)
      throw std::invalid_argument("params do not match their query shape");
    return check;
  }
  throw std::invalid_argument("tree level parameters are created by opir_tree_level_create");
}

// Allocates a handle for already checked parameters (any view); `rs` makes
// it a row shard of the layout (view OPIR_VIEW_ROW_SHARD).
opir_status create_handle(const opir_params &checked, int device, opir_server **out,
                          const opir::RowShard *rs = nullptr) {
  opir_server *s = new (std::nothrow) opir_server();
  if (!s) return OPIR_ERR_NO_MEMORY;
  const opir_status st = guarded(s, [&] {
    s->params = checked;
    s->device = device;
    if (rs) {
      s->shard = rs->shard;
      s->num_shards = rs->num_shards;
      s->host_rows = rs->rows;
    }
    DeviceGuard g(device);
    ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (is_c4(checked)) {
      s->c4.reset(new opir4::Server(checked, s->stream, rs));
      return;
    }
    setup_device_params(s);
    s->tree_h = s->shape.num_dims > 1 ? s->shape.num_dims - 1 : 0;
    if (rs) {  // the shard's rows only; MUX levels 0 .. tree_h - 1 run here
      s->tree_h = rs->tree_h;
      s->shape.other = static_cast<uint32_t>(rs->rows.size());
      s->shape.num_pt = static_cast<uint64_t>(s->shape.other) * s->shape.n0;
      s->row_map.alloc(rs->rows.size());
      ck(cudaMemcpy(s->row_map.p, rs->rows.data(), rs->rows.size() * 4, cudaMemcpyHostToDevice),
         "row map");
    }
    const opir::Shape &sh = s->shape;
    const uint64_t db_bytes = 2ull * kN * 4 * sh.other * sh.n0p;
    s->db8.alloc(db_bytes);
    ck(cudaMemsetAsync(s->db8.p, 0, db_bytes, s->stream), "db memset");
    opir::make_plane_map(&s->map_db[0], s->db8.p, sh.n0p, sh.other, 2ull * kN * 4, 128, 128);
    opir::make_plane_map(&s->map_db[1], s->db8.p, sh.n0p, sh.other, 2ull * kN * 4, 128, 64);
    s->err.alloc(1);
    ck(cudaMemsetAsync(s->err.p, 0, sizeof(uint32_t), s->stream), "err memset");
    ck(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device), "sm count");
    if (const char *gph = std::getenv("OPIR_GRAPHS")) s->use_graphs = std::strcmp(gph, "0") != 0;
    if (const char *m = std::getenv("OPIR_SCAN")) {
      if (std::strcmp(m, "tc") == 0) s->scan_mode = 1;
      else if (std::strcmp(m, "cuda") == 0) s->scan_mode = 2;
    }
    ck(cudaStreamSynchronize(s->stream), "create");
  });
  if (st != OPIR_OK) {
    opir_server_destroy(s);
    return st;
  }
  *out = s;
  return OPIR_OK;
}

void require_view(const opir_server *s, bool ok, const char *what) {
  if (!ok)
    throw std::invalid_argument(std::string(what) + " is not available on a handle created with " +
                                (s->params.view == OPIR_VIEW_QUERY_SHAPE ? "a query shape (no database)"
                                 : s->params.view == OPIR_VIEW_ROW_SHARD
                                     ? "a row shard (opir_server_make_query_shard_batch)"
                                 : s->params.view == OPIR_VIEW_LAYOUT ? "a whole layout"
                                                                      : "a tree level database"));
}
bool is_layout(const opir_server *s) { return s->params.view == OPIR_VIEW_LAYOUT; }
bool has_database(const opir_server *s) {
  return s->params.view == OPIR_VIEW_LAYOUT || s->params.view == OPIR_VIEW_ROW_SHARD;
}

// select_level on a tree level handle (single-modulus set): the alpha
// ciphertexts through the first dimension into `other` candidates, then
// fold_count MSB-first MUX steps (levels 1..fold of the handle's MUX shape,
// selector slot a = the a-th step's beta selector).
void select_fold_k1(opir_server *s, const uint64_t *alpha, const uint64_t *fold_sel,
                    uint32_t fold, uint64_t *out) {
  const opir::Shape &sh = s->shape;
  ensure_capacity(s, 1);
  DevBuf<uint64_t> in;
  const uint64_t rows_per_sel = 2ull * sh.l_ep;
  in.alloc(std::max<uint64_t>(2ull * sh.n0, fold * rows_per_sel * 2) * kN);
  ck(cudaMemcpyAsync(in.p, alpha, 2ull * sh.n0 * kN * 8, cudaMemcpyHostToDevice, s->stream), "upload");
  opir::launch_split_u64(s->dp, in.p, s->lvl[0].p, 1, 2ull * sh.n0, 0, s->stream);
  run_first_dim(s, s->lvl[0].p, 1);
  const uint32_t *res = s->mid[0].p;
  if (fold) {
    ck(cudaStreamSynchronize(s->stream), "upload");  // `in` is reused
    ck(cudaMemcpyAsync(in.p, fold_sel, fold * rows_per_sel * 2 * kN * 8, cudaMemcpyHostToDevice,
                       s->stream), "upload");
    // slot 0 of the handle's selector set is unused: step a takes slot a
    opir::launch_split_u64(s->dp, in.p, s->sel.p + rows_per_sel * kCtWords, 1,
                           fold * rows_per_sel * 2, 0, s->stream);
    for (uint32_t a = 1; a <= fold; ++a)
      opir::launch_mux_level(s->dp, sh, a, sh.num_dims - 1, s->mid[(a - 1) & 1].p, s->mid[a & 1].p,
                             sh.other, s->sel.p, 1, s->stream);
    res = s->mid[fold & 1].p;
  }
  DevBuf<uint64_t> o;
  o.alloc(2 * kN);
  opir::launch_compose_u64(s->dp, res, 0, o.p, 1, 2, s->stream);
  ck(cudaMemcpyAsync(out, o.p, 2 * kN * 8, cudaMemcpyDeviceToHost, s->stream), "download");
  ck(cudaStreamSynchronize(s->stream), "select_level");
  check_device_error(s);
}

// The client ids of a shard batch must be those of the handle's last
// make_query_shard batch: their selectors are still in the handle.
void check_shard_ids(const std::vector<uint64_t> &last, uint32_t n, const uint64_t *ids) {
  if (last.size() != n || !std::equal(last.begin(), last.end(), ids))
    throw std::invalid_argument(
        "combine_shards: client ids differ from this shard's last make_query_shard batch");
}

// The last log2 G MUX levels over the G partial ciphertexts of each query
// (d_partials: G x n x 2N u64, shard-major), then the modulus switch.
void combine_k1(opir_server *s, uint32_t n, const uint64_t *d_partials, uint64_t *d_resp) {
  const uint32_t G = s->num_shards, h = s->shape.num_dims - 1;
  const uint64_t words = static_cast<uint64_t>(n) * G * kCtWords;
  for (auto &b : s->comb)
    if (b.n < words) b.alloc(words);
  for (uint32_t g = 0; g < G; ++g)  // query i's G ciphertexts side by side
    opir::launch_split_u64(s->dp, d_partials + static_cast<uint64_t>(g) * n * 2 * kN,
                           s->comb[0].p + static_cast<uint64_t>(g) * kCtWords, n, 2,
                           static_cast<uint64_t>(G) * kCtWords, s->stream);
  int cur = 0;
  for (uint32_t a = s->tree_h; a < h; ++a, cur ^= 1)
    opir::launch_mux_level(s->dp, s->shape, a, h, s->comb[cur].p, s->comb[cur ^ 1].p, G, s->sel.p,
                           n, s->stream);
  opir::launch_modswitch(s->dp, s->comb[cur].p, G, d_resp, nullptr, resp_bytes_of(s->params), n,
                         s->stream);
}

// Orders the handle's stream after the caller's work on `user` (if any).
void wait_user(opir_server *s, cudaStream_t user) {
  if (!user) return;
  cudaEvent_t e;
  ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  ck(cudaEventRecord(e, user), "event record");
  ck(cudaStreamWaitEvent(s->stream, e, 0), "wait");
  cudaEventDestroy(e);
}
// Orders `user` (if any) after the work enqueued on the handle's stream.
void signal_user(opir_server *s, cudaStream_t user) {
  if (!user) return;
  cudaEvent_t e;
  ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  ck(cudaEventRecord(e, s->stream), "event record");
  ck(cudaStreamWaitEvent(user, e, 0), "wait");
  cudaEventDestroy(e);
}

}  // namespace

namespace {

// Times `launch` (one warm-up, then three back to back) on the handle's stream.
template <typename F>
float time_launches(opir_server *s, cudaEvent_t e0, cudaEvent_t e1, F &&launch) {
  launch();
  ck(cudaEventRecord(e0, s->stream), "event record");
  for (int r = 0; r < 3; ++r) launch();
  ck(cudaEventRecord(e1, s->stream), "event record");
  ck(cudaEventSynchronize(e1), "autotune");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, e0, e1), "event time");
  return ms;
}

// Cluster width of every expansion level (1, 2, 4, 8 CTAs per key switch)
// and MUX level (1, 2, 4 CTAs per MUX) per batch bucket: each width timed on
// the handle's scratch buffers with zero ciphertexts and zero key rows (the
// kernels' work does not depend on the values), the fastest kept. Every
// width computes the same result bit for bit.
void tune_levels(opir_server *s, uint32_t max_batch, cudaEvent_t e0, cudaEvent_t e1) {
  const opir::Shape base = s->shape;
  const uint64_t bv_words = std::max<uint64_t>(1, static_cast<uint64_t>(base.h) * base.l_ks * 4 * kN);
  const uint64_t gsw_words = 2ull * base.l_key * 4 * kN;
  DevBuf<uint32_t> zkeys;
  zkeys.alloc(bv_words + gsw_words);
  ck(cudaMemsetAsync(zkeys.p, 0, zkeys.n * 4, s->stream), "memset");
  for (auto *b : {&s->lvl[0], &s->lvl[1], &s->mid[0], &s->mid[1], &s->sel})
    ck(cudaMemsetAsync(b->p, 0, b->n * 4, s->stream), "memset");
  std::vector<const uint32_t *> ptrs(2ull * max_batch);
  for (uint32_t i = 0; i < max_batch; ++i) {
    ptrs[i] = zkeys.p;
    ptrs[max_batch + i] = zkeys.p + bv_words;
  }
  ck(cudaMemcpyAsync(s->keyptrs.p, ptrs.data(), ptrs.size() * sizeof(void *), cudaMemcpyHostToDevice,
                     s->stream), "key pointers");
  const uint64_t bv_level_stride = static_cast<uint64_t>(base.l_ks) * 4 * kN;
  for (int b = 0; b < kTileBuckets; ++b) {
    const uint32_t n = std::min<uint32_t>(1u << b, max_batch);
    LevelSplits ls;
    for (uint32_t d = 0; d < base.h && d < 16; ++d) {
      float best = 1e30f;
      for (uint8_t c : {1, 2, 4, 8}) {
        opir::Shape sh = base;
        sh.split_exp[d] = c;
        const float ms = time_launches(s, e0, e1, [&] {
          opir::launch_expand_level(s->dp, sh, d, s->lvl[d & 1].p, s->lvl_slots,
                                    s->lvl[(d + 1) & 1].p, s->lvl_slots, s->keyptrs.p,
                                    bv_level_stride, n, s->stream);
        });
        if (ms < best) { best = ms; ls.exp[d] = c; }
      }
    }
    for (uint32_t a = 0; a < s->tree_h && a < 32; ++a) {
      float best = 1e30f;
      for (uint8_t c : {1, 2, 4}) {
        if (c == 4 && base.l_ep % 2 != 0) continue;  // digits do not halve
        opir::Shape sh = base;
        sh.split_mux[a] = c;
        const float ms = time_launches(s, e0, e1, [&] {
          opir::launch_mux_level(s->dp, sh, a, s->tree_h, s->mid[a & 1].p, s->mid[(a + 1) & 1].p,
                                 base.other, s->sel.p, n, s->stream);
        });
        if (ms < best) { best = ms; ls.mux[a] = c; }
      }
    }
    s->split[b] = ls;
    if (n == max_batch) break;
  }
  ck(cudaStreamSynchronize(s->stream), "autotune");
  clear_graphs(s);
}

// Device rate of a register-resident probe kernel: one warm-up launch, then
// three timed launches on a private stream; `launch(sink, st)` returns the
// units (butterflies, outputs) one launch performs.
template <class F>
double probe_rate(int device, size_t sink_words, F &&launch) {
  DeviceGuard g(device);
  DevBuf<uint64_t> sink;
  sink.alloc(sink_words);
  cudaStream_t st = nullptr;
  ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double rate = 0;
  try {
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    launch(sink.p, st);  // warm-up
    ck(cudaEventRecord(e0, st), "event record");
    uint64_t units = 0;
    for (int r = 0; r < 3; ++r) units += launch(sink.p, st);
    ck(cudaEventRecord(e1, st), "event record");
    ck(cudaEventSynchronize(e1), "probe");
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, e0, e1), "event time");
    rate = static_cast<double>(units) / (static_cast<double>(ms) / 1e3);
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return rate;
}

}  // namespace

extern "C" {

const char *opir_version(void) { return "onionpir_b200 0.1 (sm_100a)"; }

opir_status opir_params_init(const opir_layout *layout, opir_params *out) {
  if (!layout || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] { *out = opir::derive_params(*layout); });
}

opir_status opir_params_init_config(opir_config config, const opir_layout *layout,
                                    opir_params *out) {
  if (!layout || !out) return OPIR_ERR_INVALID_ARGUMENT;
  if (config == OPIR_CONFIG_N2048_K1_COMP) return opir_params_init(layout, out);
  if (config == OPIR_CONFIG_N2048_K2_MP)
    return guarded(nullptr, [&] { *out = opir::derive_params_k2mp(*layout); });
  if (config == OPIR_CONFIG_N2048_K1)
    return guarded(nullptr, [&] { *out = opir::derive_params_k1p(*layout); });
  if (config != OPIR_CONFIG_N4096_K2_MP) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] { *out = opir4::derive(*layout); });
}

size_t opir_response_bytes(const opir_params *params) {
  return params ? resp_bytes_of(*params) : 0;
}

opir_status opir_server_create(const opir_params *params, int device, opir_server **out) {
  if (!params || !out) return OPIR_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  opir_params checked{};
  const opir_status vs = guarded(nullptr, [&] { checked = checked_params(*params); });
  if (vs != OPIR_OK) return vs;
  return create_handle(checked, device, out);
}

void opir_server_destroy(opir_server *s) {
  if (!s) return;
  {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    clear_graphs(s);
    s->c4.reset();
    s->clients.clear();
    s->tables.reset();
    s->db8.reset();
    s->err.reset();
    s->q_u64.reset();
    s->resp_u64.reset();
    s->resp_bytes.reset();
    for (auto &b : s->lvl) b.reset();
    s->sel.reset();
    s->qb.reset();
    s->cmat.reset();
    for (auto &b : s->mid) b.reset();
    s->keyptrs.reset();
    for (KeyPtrSlot &sl : s->kp_ring) {
      if (sl.host) cudaFreeHost(sl.host);
      if (sl.done) cudaEventDestroy(sl.done);
    }
    for (auto &evs : s->ev_pool)
      for (auto &e : evs) cudaEventDestroy(e);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (prev >= 0) cudaSetDevice(prev);
  }
  delete s;
}

const char *opir_server_last_error(const opir_server *s) {
  return s ? s->last_error.c_str() : "null server handle";
}

opir_status opir_server_params(const opir_server *s, opir_params *out) {
  if (!s || !out) return OPIR_ERR_INVALID_ARGUMENT;
  *out = s->params;
  return OPIR_OK;
}

opir_status opir_server_load_db_u16(opir_server *s, uint64_t logical, const uint16_t *coeffs) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    require_view(s, has_database(s), "load_data");
    if (!coeffs && logical) throw std::invalid_argument("PirServer::load_data requires a source");
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->load_db_u16(logical, coeffs);
    const uint64_t t = s->params.plain_mod;
    load_tiles(s, logical, [&](uint64_t b, uint64_t e, uint16_t *dst) {
      const uint16_t *src = coeffs + b * kN;
      for (uint64_t i = 0; i < (e - b) * kN; ++i) {
        if (src[i] >= t)
          throw std::invalid_argument("Plaintext source coefficient exceeds the plaintext modulus");
        dst[i] = src[i];
      }
    });
  });
}

opir_status opir_server_load_db(opir_server *s, uint64_t logical, const uint64_t *coeffs) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    require_view(s, has_database(s), "load_data");
    if (!coeffs && logical) throw std::invalid_argument("PirServer::load_data requires a source");
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->load_db(logical, coeffs);
    const uint64_t t = s->params.plain_mod;
    load_tiles(s, logical, [&](uint64_t b, uint64_t e, uint16_t *dst) {
      const uint64_t *src = coeffs + b * kN;
      for (uint64_t i = 0; i < (e - b) * kN; ++i) {
        if (src[i] >= t)
          throw std::invalid_argument("Plaintext source coefficient exceeds the plaintext modulus");
        dst[i] = static_cast<uint16_t>(src[i]);
      }
    });
  });
}

opir_status opir_server_load_db_source(opir_server *s, uint64_t logical,
                                       opir_plaintext_source source, void *user) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    require_view(s, has_database(s), "load_data");
    if (!source) throw std::invalid_argument("PirServer::load_data requires a source");
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->load_db_source(logical, source, user);
    const uint64_t t = s->params.plain_mod;
    std::vector<uint64_t> pt(kN);
    load_tiles(s, logical, [&](uint64_t b, uint64_t e, uint16_t *dst) {
      for (uint64_t idx = b; idx < e; ++idx) {
        if (source(user, idx, pt.data()) != 0)
          throw std::invalid_argument("Plaintext source failed");
        for (int c = 0; c < kN; ++c) {
          if (pt[c] >= t)
            throw std::invalid_argument("Plaintext source coefficient exceeds the plaintext modulus");
          dst[(idx - b) * kN + c] = static_cast<uint16_t>(pt[c]);
        }
      }
    });
  });
}

opir_status opir_server_load_db_seeded(opir_server *s, uint64_t logical, uint64_t seed) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    require_view(s, has_database(s), "load_data");
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->load_db_seeded(logical, seed);
    const opir_params &p = s->params;
    if (logical > p.num_pt)
      throw std::invalid_argument("PirServer::load_data logical plaintext count exceeds its layout");
    s->db_loaded = false;
    const uint64_t chunk = 1ull << 20;
    const uint64_t local_pt = static_cast<uint64_t>(s->shape.other) * s->shape.n0;
    for (uint64_t pb = 0; pb < local_pt; pb += chunk)
      opir::launch_db_preprocess(s->dp, s->shape, nullptr, 0, seed, p.plain_mod, logical, pb,
                                 std::min<uint64_t>(local_pt, pb + chunk), s->row_map.p, s->db8.p,
                                 s->stream);
    ck(cudaStreamSynchronize(s->stream), "db preprocess");
    s->db_loaded = true;
  });
}

opir_status opir_server_set_client_keys(opir_server *s, uint64_t client_id,
                                        const uint64_t *bv_keys, const uint32_t *galois_ks,
                                        uint32_t n_keys, const uint64_t *gsw_key) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (s->c4) {
      DeviceGuard g(s->device);
      return s->c4->set_client_keys(client_id, bv_keys, galois_ks, n_keys, gsw_key);
    }
    const opir_params &p = s->params;
    const uint32_t h = p.expansion_height;
    if (!gsw_key) throw std::invalid_argument("PirServer session key bundle cannot be null");
    if (n_keys < h) throw std::invalid_argument("PirServer session lacks keys for its expansion height");
    if (n_keys && (!bv_keys || !galois_ks)) throw std::invalid_argument("null BV key arrays");
    const uint64_t pw = poly_words(p);
    const size_t key_words = static_cast<size_t>(p.l_ks) * 2 * pw;  // one BvKeySwitchKey, u64
    std::vector<uint64_t> ordered(static_cast<size_t>(h) * key_words);
    for (uint32_t d = 0; d < h; ++d) {
      const uint32_t want = kN / (1u << d) + 1;
      int found = -1;
      for (uint32_t i = 0; i < n_keys; ++i)
        if (galois_ks[i] == want) { found = static_cast<int>(i); break; }
      if (found < 0) throw std::out_of_range("BvGaloisKeys::get: galois_k not found");
      std::memcpy(ordered.data() + d * key_words, bv_keys + found * key_words, key_words * 8);
    }
    const size_t gsw_words = static_cast<size_t>(2) * p.l_key * 2 * pw;
    if (is_k2mp(p)) {  // limb-major rows: limb (i / N) % 2
      const uint64_t m[2] = {p.q1, p.q2};
      for (size_t i = 0; i < ordered.size(); ++i)
        if (ordered[i] >= m[(i / kN) & 1]) throw std::invalid_argument("BV key value not reduced mod its limb");
      for (size_t i = 0; i < gsw_words; ++i)
        if (gsw_key[i] >= m[(i / kN) & 1]) throw std::invalid_argument("RGSW key value not reduced mod its limb");
    } else {
      for (uint64_t v : ordered)
        if (v >= p.q) throw std::invalid_argument("BV key value not reduced mod q");
      for (size_t i = 0; i < gsw_words; ++i)
        if (gsw_key[i] >= p.q) throw std::invalid_argument("RGSW key value not reduced mod q");
    }
    DeviceGuard g(s->device);
    ClientKeys k;
    DevBuf<uint64_t> tmp;
    tmp.alloc(std::max(ordered.size(), gsw_words));
    k.bv.alloc(std::max<size_t>(1, ordered.size() / pw * 2 * kN));
    k.gsw.alloc(gsw_words / pw * 2 * kN);
    if (!ordered.empty()) {
      ck(cudaMemcpyAsync(tmp.p, ordered.data(), ordered.size() * 8, cudaMemcpyHostToDevice, s->stream), "bv upload");
      opir::launch_split_u64(s->dp, tmp.p, k.bv.p, 1, ordered.size() / pw, 0, s->stream);
      ck(cudaStreamSynchronize(s->stream), "bv split");
    }
    ck(cudaMemcpyAsync(tmp.p, gsw_key, gsw_words * 8, cudaMemcpyHostToDevice, s->stream), "gsw upload");
    opir::launch_split_u64(s->dp, tmp.p, k.gsw.p, 1, gsw_words / pw, 0, s->stream);
    ck(cudaStreamSynchronize(s->stream), "gsw split");
    ClientKeys &slot = s->clients[client_id];
    std::swap(slot.bv.p, k.bv.p); std::swap(slot.bv.n, k.bv.n);
    std::swap(slot.gsw.p, k.gsw.p); std::swap(slot.gsw.n, k.gsw.n);
  });
}

opir_status opir_server_set_client_keys_ex(opir_server *s, uint64_t client_id,
                                           const uint64_t *bv_keys, const uint32_t *galois_ks,
                                           uint32_t n_keys, const uint64_t *gsw_key,
                                           uint32_t key_form) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  if (key_form == OPIR_KEYS_NTT)
    return opir_server_set_client_keys(s, client_id, bv_keys, galois_ks, n_keys, gsw_key);
  std::vector<uint64_t> bv, gsw;
  const opir_status st = guarded(s, [&] {
    if (key_form != OPIR_KEYS_COEFF) throw std::invalid_argument("unknown key form");
    if (!gsw_key) throw std::invalid_argument("PirServer session key bundle cannot be null");
    if (n_keys && (!bv_keys || !galois_ks)) throw std::invalid_argument("null BV key arrays");
    const opir_params &p = s->params;
    const uint32_t n = p.poly_degree, K = p.num_limbs;
    const uint64_t mods[2] = {K == 1 ? p.q : p.q1, K == 1 ? 0 : p.q2};
    const size_t key_words = static_cast<size_t>(p.l_ks) * 2 * K * n;
    const size_t gsw_words = static_cast<size_t>(2) * p.l_key * 2 * K * n;
    bv.assign(bv_keys, bv_keys + n_keys * key_words);
    gsw.assign(gsw_key, gsw_key + gsw_words);
    for (const std::vector<uint64_t> *v : {&bv, &gsw})
      for (size_t i = 0; i < v->size(); ++i)
        if ((*v)[i] >= mods[(i / n) % K]) throw std::invalid_argument("key value not reduced mod its limb");
    // coefficient form -> this library's NTT domain, on the device
    DeviceGuard g(s->device);
    const std::vector<uint64_t> fw = opir::forward_twiddles(p);
    DevBuf<uint64_t> d_fw, d;
    d_fw.alloc(fw.size());
    d.alloc(bv.size() + gsw.size());
    ck(cudaMemcpyAsync(d_fw.p, fw.data(), fw.size() * 8, cudaMemcpyHostToDevice, s->stream), "twiddle upload");
    if (!bv.empty())
      ck(cudaMemcpyAsync(d.p, bv.data(), bv.size() * 8, cudaMemcpyHostToDevice, s->stream), "bv upload");
    ck(cudaMemcpyAsync(d.p + bv.size(), gsw.data(), gsw.size() * 8, cudaMemcpyHostToDevice, s->stream),
       "gsw upload");
    opir::forward_ntt_polys(d.p, (bv.size() + gsw.size()) / n, p, d_fw.p, s->stream);
    if (!bv.empty())
      ck(cudaMemcpyAsync(bv.data(), d.p, bv.size() * 8, cudaMemcpyDeviceToHost, s->stream), "bv download");
    ck(cudaMemcpyAsync(gsw.data(), d.p + bv.size(), gsw.size() * 8, cudaMemcpyDeviceToHost, s->stream),
       "gsw download");
    ck(cudaStreamSynchronize(s->stream), "key NTT");
  });
  if (st != OPIR_OK) return st;
  return opir_server_set_client_keys(s, client_id, bv.empty() ? nullptr : bv.data(), galois_ks,
                                     n_keys, gsw.data());
}

opir_status opir_server_remove_client(opir_server *s, uint64_t client_id) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->remove_client(client_id);
    ck(cudaStreamSynchronize(s->stream), "remove_client");
    if (s->clients.erase(client_id) == 0) throw std::out_of_range("unknown client id");
  });
}

opir_status opir_server_make_query_batch(opir_server *s, uint32_t n, const uint64_t *client_ids,
                                         const uint64_t *queries, uint64_t *responses) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (n && (!client_ids || !queries || !responses)) throw std::invalid_argument("null argument");
    require_view(s, is_layout(s), "make_query");
    if (s->c4) {
      DeviceGuard g(s->device);
      return s->c4->make_query_batch(n, client_ids, queries, responses, c4_events(s));
    }
    const uint64_t pw = poly_words(s->params);
    check_query_values(s, queries, static_cast<size_t>(n) * 2 * pw);
    DeviceGuard g(s->device);
    ensure_capacity(s, n);
    ck(cudaMemcpyAsync(s->q_u64.p, queries, static_cast<size_t>(n) * 2 * pw * 8,
                       cudaMemcpyHostToDevice, s->stream), "query upload");
    run_pipeline(s, client_ids, n, s->q_u64.p, s->resp_u64.p, nullptr);
    ck(cudaMemcpyAsync(responses, s->resp_u64.p, static_cast<size_t>(n) * 2 * kN * 8,
                       cudaMemcpyDeviceToHost, s->stream), "response download");
    finish(s);
  });
}

opir_status opir_server_make_query(opir_server *s, uint64_t client_id, const uint64_t *query,
                                   uint64_t *response) {
  return opir_server_make_query_batch(s, 1, &client_id, query, response);
}

opir_status opir_server_make_query_batch_device(opir_server *s, uint32_t n,
                                                const uint64_t *client_ids,
                                                const uint64_t *d_queries, uint64_t *d_responses,
                                                void *stream) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (n && (!client_ids || !d_queries || !d_responses)) throw std::invalid_argument("null argument");
    require_view(s, is_layout(s), "make_query");
    DeviceGuard g(s->device);
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    wait_user(s, user);  // order after the caller's prior work on its stream
    if (s->c4)
      s->c4->make_query_batch_device(n, client_ids, d_queries, d_responses, c4_events(s));
    else
      run_pipeline(s, client_ids, n, d_queries, d_responses, nullptr);
    signal_user(s, user);
  });
}

// ---------------------------------------------------------------- row shards

opir_status opir_row_shard_rows(const opir_params *params, uint32_t shard, uint32_t num_shards,
                                uint32_t *rows, uint64_t *n_rows, uint32_t *tree_h) {
  if (!params || !n_rows) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    const opir_params p = checked_params(*params);
    if (p.view != OPIR_VIEW_LAYOUT) throw std::invalid_argument("row shards split a database layout");
    const opir::RowShard rs = opir::row_shard(p.other_dim_sz, p.num_dims, shard, num_shards);
    if (rows) std::copy(rs.rows.begin(), rs.rows.end(), rows);
    *n_rows = rs.rows.size();
    if (tree_h) *tree_h = rs.tree_h;
  });
}

opir_status opir_server_create_row_shard(const opir_params *params, uint32_t shard,
                                         uint32_t num_shards, int device, opir_server **out) {
  if (!params || !out) return OPIR_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  opir_params checked{};
  opir::RowShard rs;
  const opir_status vs = guarded(nullptr, [&] {
    checked = checked_params(*params);
    if (checked.view != OPIR_VIEW_LAYOUT)
      throw std::invalid_argument("row shards split a database layout");
    if (is_k2mp(checked) || is_k1p(checked))
      throw std::invalid_argument(
          "row shards are built for CONFIG_N2048_K1_COMP and CONFIG_N4096_K2_MP");
    rs = opir::row_shard(checked.other_dim_sz, checked.num_dims, shard, num_shards);
    checked.view = OPIR_VIEW_ROW_SHARD;
  });
  if (vs != OPIR_OK) return vs;
  return create_handle(checked, device, out, &rs);
}

opir_status opir_server_make_query_shard_batch(opir_server *s, uint32_t n,
                                               const uint64_t *client_ids,
                                               const uint64_t *queries, uint64_t *partials) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (n && (!client_ids || !queries || !partials)) throw std::invalid_argument("null argument");
    require_view(s, is_row_shard(s), "make_query_shard");
    DeviceGuard g(s->device);
    if (s->c4) {
      s->c4->make_query_batch(n, client_ids, queries, partials, c4_events(s));
    } else {
      check_query_values(s, queries, static_cast<size_t>(n) * 2 * kN);
      ensure_capacity(s, n);
      ck(cudaMemcpyAsync(s->q_u64.p, queries, static_cast<size_t>(n) * 2 * kN * 8,
                         cudaMemcpyHostToDevice, s->stream), "query upload");
      run_pipeline(s, client_ids, n, s->q_u64.p, s->resp_u64.p, nullptr);
      ck(cudaMemcpyAsync(partials, s->resp_u64.p, static_cast<size_t>(n) * 2 * kN * 8,
                         cudaMemcpyDeviceToHost, s->stream), "partial download");
      finish(s);
    }
    s->shard_ids.assign(client_ids, client_ids + n);
  });
}

opir_status opir_server_make_query_shard_batch_device(opir_server *s, uint32_t n,
                                                      const uint64_t *client_ids,
                                                      const uint64_t *d_queries,
                                                      uint64_t *d_partials, void *stream) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (n && (!client_ids || !d_queries || !d_partials)) throw std::invalid_argument("null argument");
    require_view(s, is_row_shard(s), "make_query_shard");
    DeviceGuard g(s->device);
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    wait_user(s, user);
    if (s->c4)
      s->c4->make_query_batch_device(n, client_ids, d_queries, d_partials, c4_events(s));
    else
      run_pipeline(s, client_ids, n, d_queries, d_partials, nullptr);
    s->shard_ids.assign(client_ids, client_ids + n);
    signal_user(s, user);
  });
}

opir_status opir_server_combine_shards(opir_server *s, uint32_t n, const uint64_t *client_ids,
                                       const uint64_t *partials, uint64_t *responses) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (n && (!client_ids || !partials || !responses)) throw std::invalid_argument("null argument");
    require_view(s, is_row_shard(s), "combine_shards");
    check_shard_ids(s->shard_ids, n, client_ids);
    if (n == 0) return;
    DeviceGuard g(s->device);
    const size_t ct = s->c4 ? 4ull * s->params.poly_degree : 2ull * kN;
    const size_t words = static_cast<size_t>(s->num_shards) * n * ct;
    if (s->c4) {
      s->c4->combine_host(n, partials, responses);
      return;
    }
    check_query_values(s, partials, words);
    DevBuf<uint64_t> d_in, d_out;
    d_in.alloc(words);
    d_out.alloc(static_cast<size_t>(n) * 2 * kN);
    ck(cudaMemcpyAsync(d_in.p, partials, words * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    combine_k1(s, n, d_in.p, d_out.p);
    ck(cudaMemcpyAsync(responses, d_out.p, static_cast<size_t>(n) * 2 * kN * 8,
                       cudaMemcpyDeviceToHost, s->stream), "download");
    finish(s);
  });
}

opir_status opir_server_combine_shards_device(opir_server *s, uint32_t n,
                                              const uint64_t *client_ids,
                                              const uint64_t *d_partials, uint64_t *d_responses,
                                              void *stream) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (n && (!client_ids || !d_partials || !d_responses)) throw std::invalid_argument("null argument");
    require_view(s, is_row_shard(s), "combine_shards");
    check_shard_ids(s->shard_ids, n, client_ids);
    if (n == 0) return;
    DeviceGuard g(s->device);
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    wait_user(s, user);
    if (s->c4)
      s->c4->combine_device(n, d_partials, d_responses);
    else
      combine_k1(s, n, d_partials, d_responses);
    signal_user(s, user);
  });
}

opir_status opir_server_set_priority(opir_server *s, int priority) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    DeviceGuard g(s->device);
    int least = 0, greatest = 0;
    ck(cudaDeviceGetStreamPriorityRange(&least, &greatest), "priority range");
    const int p = std::min(std::max(priority, greatest), least);  // greatest < least
    cudaStream_t ns = nullptr;
    ck(cudaStreamCreateWithPriority(&ns, cudaStreamNonBlocking, p), "cudaStreamCreateWithPriority");
    ck(cudaStreamSynchronize(s->stream), "set_priority");
    if (s->c4) s->c4->set_stream(ns);
    cudaStreamDestroy(s->stream);
    s->stream = ns;
  });
}

opir_status opir_server_set_scan_wait_limit(opir_server *s, uint64_t cycles) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    DeviceGuard g(s->device);
    if (cycles > (1ull << 40)) throw std::invalid_argument("wait limit above 2^40 cycles");
    const long long c = static_cast<long long>(cycles);
    ck(cudaStreamSynchronize(s->stream), "set_scan_wait_limit");
    if (s->c4) return s->c4->set_scan_wait_limit(c);
    if (c != s->scan_wait) clear_graphs(s);  // captured scans hold the old limit
    s->scan_wait = c;
  });
}

opir_status opir_plan_memory(const opir_params *params, opir_memory_plan *out) {
  if (!params || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    if (is_c4(*params)) return opir4::Server::plan_memory(*params, out);
    if (!is_k2mp(*params) &&
        (params->poly_degree != static_cast<uint32_t>(kN) || params->num_limbs != 1))
      throw std::invalid_argument(
          "unsupported parameter set (CONFIG_N2048_K1_COMP, CONFIG_N2048_K2_MP or CONFIG_N4096_K2_MP)");
    uint64_t slots = 0;
    const opir::Shape sh = make_shape(*params, &slots);
    const uint32_t rb = resp_bytes_of(*params);
    const uint64_t pw = poly_words(*params);
    const uint64_t one = plan_scratch(sh, slots, rb, 1, pw).bytes();
    const uint64_t two = plan_scratch(sh, slots, rb, 2, pw).bytes();
    out->database_bytes = 2ull * kN * 4 * sh.other * sh.n0p + 16ull * kN * 4 + sizeof(uint32_t);
    out->client_key_bytes =
        (static_cast<uint64_t>(sh.h) * sh.l_ks * 2 * kN + 2ull * sh.l_key * 2 * kN) * 2 * 4;
    out->scratch_bytes_per_query = two - one;
    out->scratch_bytes_fixed = 2 * one - two;
  });
}

opir_status opir_server_reserve(opir_server *s, uint32_t max_batch) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->reserve(max_batch);
    ensure_capacity(s, max_batch);
    grow_keyptr_slots(s, 2ull * max_batch);
  });
}

opir_status opir_server_autotune(opir_server *s, uint32_t max_batch) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (!(s->c4 ? s->c4->db_loaded() : s->db_loaded))
      throw std::runtime_error("autotune before load_data");
    if (max_batch == 0) throw std::invalid_argument("max_batch must be positive");
    if (s->c4) return;  // the 64-bit-limb scan has no tiling to tune
    DeviceGuard g(s->device);
    ensure_capacity(s, max_batch);
    grow_keyptr_slots(s, 2ull * max_batch);
    if (s->shape.n0p > 8192) {  // the CUDA-core scan has no tiling to tune
      cudaEvent_t e0, e1;
      ck(cudaEventCreate(&e0), "event");
      ck(cudaEventCreate(&e1), "event");
      try {
        tune_levels(s, max_batch, e0, e1);
      } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return;
    }
    std::vector<ScanTile> cands;
    for (uint32_t kt : {128u, 64u})
      for (uint32_t nt : {16u, 32u, 64u}) {
        const uint32_t hi = opir::scan_tc_max_stages(nt, kt);
        for (uint32_t st = std::max(2u, hi > 2 ? hi - 1 : 2u); st <= hi; ++st) cands.push_back({nt, kt, st});
      }
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    try {
      for (int b = 0; b < kTileBuckets; ++b) {
        const uint32_t n = std::min<uint32_t>(1u << b, max_batch);
        float best = 1e30f;
        for (const ScanTile &c : cands) {
          if (c.ntile > 16 && 2 * n <= c.ntile / 2) continue;  // mostly empty tiles
          launch_scan_tc_tile(s, n, c);
          ck(cudaEventRecord(e0, s->stream), "event record");
          for (int r = 0; r < 3; ++r) launch_scan_tc_tile(s, n, c);
          ck(cudaEventRecord(e1, s->stream), "event record");
          ck(cudaEventSynchronize(e1), "autotune");
          float ms = 0;
          ck(cudaEventElapsedTime(&ms, e0, e1), "event time");
          if (ms < best) { best = ms; s->tile[b] = c; }
          clear_graphs(s);
        }
        check_device_error(s);
        if (n == max_batch) break;
      }
      tune_levels(s, max_batch, e0, e1);
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  });
}

opir_status opir_server_level_splits(const opir_server *s, uint32_t n, uint8_t *expand,
                                     uint8_t *mux) {
  if (!s || !expand || !mux || n == 0) return OPIR_ERR_INVALID_ARGUMENT;
  if (s->c4) {  // the 64-bit-limb levels have fixed widths
    std::fill(expand, expand + 16, 0);
    std::fill(mux, mux + 32, 0);
    return OPIR_OK;
  }
  const LevelSplits &ls = s->split[tile_bucket(n)];
  std::copy(std::begin(ls.exp), std::end(ls.exp), expand);
  std::copy(std::begin(ls.mux), std::end(ls.mux), mux);
  return OPIR_OK;
}

opir_status opir_server_scan_tile(const opir_server *s, uint32_t n, uint32_t *ntile, uint32_t *kt,
                                  uint32_t *stages) {
  if (!s || !ntile || !kt || !stages || n == 0) return OPIR_ERR_INVALID_ARGUMENT;
  if (s->c4) {  // CUDA-core scan: no tensor-core tiling
    *ntile = *kt = *stages = 0;
    return OPIR_OK;
  }
  const ScanTile t = effective_tile(s, n);
  *ntile = t.ntile;
  *kt = t.kt;
  *stages = t.stages;
  return OPIR_OK;
}

opir_status opir_server_set_stage_timing(opir_server *s, int enabled) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  s->timing = enabled != 0;
  s->timed_calls = 0;
  return OPIR_OK;
}

opir_status opir_server_stage_times(opir_server *s, float *ms_out, uint32_t *calls) {
  if (!s || !ms_out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    DeviceGuard g(s->device);
    ck(cudaStreamSynchronize(s->stream), "stage_times");
    double sum[kStages + 1] = {0, 0, 0, 0, 0, 0};
    for (uint32_t c = 0; c < s->timed_calls; ++c) {
      const cudaEvent_t *e = s->ev_pool[c].data();
      float ms = 0;
      for (int i = 0; i < kStages; ++i) {
        ck(cudaEventElapsedTime(&ms, e[i], e[i + 1]), "cudaEventElapsedTime");
        sum[i] += ms;
      }
      ck(cudaEventElapsedTime(&ms, e[kStages + 1], e[kStages + 2]), "cudaEventElapsedTime");
      sum[kStages] += ms;
    }
    for (int i = 0; i <= kStages; ++i)
      ms_out[i] = s->timed_calls ? static_cast<float>(sum[i] / s->timed_calls) : 0.f;
    if (calls) *calls = s->timed_calls;
  });
}

uint64_t opir_launch_count(void) { return opir::launch_count() + opir4::launch_count(); }

opir_status opir_server_expand_query(opir_server *s, uint64_t client_id, const uint64_t *query,
                                     uint64_t *out) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (!query || !out) throw std::invalid_argument("null argument");
    require_view(s, s->params.view != OPIR_VIEW_MATRIX, "expand_query");
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->expand_query(client_id, query, out);
    const uint64_t pw = poly_words(s->params);
    check_query_values(s, query, 2 * pw);
    ensure_capacity(s, 1);
    upload_keyptrs(s, &client_id, 1);
    ck(cudaMemcpyAsync(s->q_u64.p, query, 2 * pw * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    opir::launch_split_u64(s->dp, s->q_u64.p, s->lvl[0].p, 1, 2, 0, s->stream);
    const uint32_t *leaves = run_expand(s, 1);
    DevBuf<uint64_t> o;
    o.alloc(static_cast<size_t>(s->shape.useful) * 2 * pw);
    opir::launch_compose_u64(s->dp, leaves, 0, o.p, 1, 2ull * s->shape.useful, s->stream);
    ck(cudaMemcpyAsync(out, o.p, o.n * 8, cudaMemcpyDeviceToHost, s->stream), "download");
    ck(cudaStreamSynchronize(s->stream), "expand_query");
  });
}

opir_status opir_server_complete_selectors(opir_server *s, uint64_t client_id,
                                           const uint64_t *expanded, uint64_t *out) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (!expanded || !out) throw std::invalid_argument("null argument");
    require_view(s, s->params.view != OPIR_VIEW_MATRIX, "complete_selectors");
    if (s->c4) {
      DeviceGuard g(s->device);
      return s->c4->complete_selectors(client_id, expanded, out);
    }
    const opir::Shape &sh = s->shape;
    const uint64_t pw = poly_words(s->params);
    check_query_values(s, expanded, static_cast<size_t>(sh.useful) * 2 * pw);
    DeviceGuard g(s->device);
    ensure_capacity(s, 1);
    upload_keyptrs(s, &client_id, 1);
    const uint32_t nsel = sh.num_dims - 1;
    if (nsel == 0) return;
    DevBuf<uint64_t> in;
    in.alloc(static_cast<size_t>(sh.useful) * 2 * pw);
    ck(cudaMemcpyAsync(in.p, expanded, in.n * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    opir::launch_split_u64(s->dp, in.p, s->lvl[0].p, 1, 2ull * sh.useful, 0, s->stream);
    opir::launch_selectors(s->dp, sh, s->lvl[0].p, s->lvl_slots, s->keyptrs.p + 1, s->sel.p, 1,
                           s->stream);
    const uint64_t polys = 2ull * nsel * 2 * sh.l_ep;
    DevBuf<uint64_t> o;
    o.alloc(polys * pw);
    opir::launch_compose_u64(s->dp, s->sel.p, 0, o.p, 1, polys, s->stream);
    ck(cudaMemcpyAsync(out, o.p, o.n * 8, cudaMemcpyDeviceToHost, s->stream), "download");
    ck(cudaStreamSynchronize(s->stream), "complete_selectors");
  });
}

opir_status opir_server_evaluate_first_dim(opir_server *s, const uint64_t *fst_query, uint64_t *out) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (!fst_query || !out) throw std::invalid_argument("null argument");
    require_view(s, is_layout(s), "evaluate_first_dim");
    if (s->c4) {
      DeviceGuard g(s->device);
      return s->c4->evaluate_first_dim(fst_query, out);
    }
    if (!s->db_loaded) throw std::runtime_error("evaluate_first_dim before load_data");
    const opir::Shape &sh = s->shape;
    const uint64_t pw = poly_words(s->params);
    check_query_values(s, fst_query, static_cast<size_t>(sh.n0) * 2 * pw);
    DeviceGuard g(s->device);
    ensure_capacity(s, 1);
    DevBuf<uint64_t> in;
    in.alloc(static_cast<size_t>(sh.n0) * 2 * pw);
    ck(cudaMemcpyAsync(in.p, fst_query, in.n * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    opir::launch_split_u64(s->dp, in.p, s->lvl[0].p, 1, 2ull * sh.n0, 0, s->stream);
    run_first_dim(s, s->lvl[0].p, 1);
    DevBuf<uint64_t> o;
    o.alloc(static_cast<size_t>(sh.other) * 2 * pw);
    opir::launch_compose_u64(s->dp, s->mid[0].p, 0, o.p, 1, 2ull * sh.other, s->stream);
    ck(cudaMemcpyAsync(out, o.p, o.n * 8, cudaMemcpyDeviceToHost, s->stream), "download");
    ck(cudaStreamSynchronize(s->stream), "evaluate_first_dim");
  });
}

opir_status opir_server_evaluate_other_dim(opir_server *s, const uint64_t *mid,
                                           const uint64_t *selectors, uint64_t *out) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    require_view(s, is_layout(s), "evaluate_other_dim");
    if (s->c4) {
      const uint32_t nsel = s->params.num_dims - 1;
      if (!mid || !out || (nsel && !selectors)) throw std::invalid_argument("null argument");
      DeviceGuard g(s->device);
      return s->c4->evaluate_other_dim(mid, selectors, out);
    }
    const opir::Shape &sh = s->shape;
    const uint32_t nsel = sh.num_dims - 1;
    if (!mid || !out || (nsel && !selectors)) throw std::invalid_argument("null argument");
    if (nsel && sh.other < (1u << (nsel - 1)))
      throw std::invalid_argument("evaluate_other_dim: layout has fewer candidates than its selector tree");
    const uint64_t pw = poly_words(s->params);
    check_query_values(s, mid, static_cast<size_t>(sh.other) * 2 * pw);
    DeviceGuard g(s->device);
    ensure_capacity(s, 1);
    DevBuf<uint64_t> in;
    const uint64_t sel_polys = 2ull * nsel * 2 * sh.l_ep;
    in.alloc(std::max<uint64_t>(static_cast<uint64_t>(sh.other) * 2, sel_polys) * pw);
    ck(cudaMemcpyAsync(in.p, mid, static_cast<size_t>(sh.other) * 2 * pw * 8,
                       cudaMemcpyHostToDevice, s->stream), "upload");
    opir::launch_split_u64(s->dp, in.p, s->mid[0].p, 1, 2ull * sh.other, 0, s->stream);
    if (nsel) {
      ck(cudaStreamSynchronize(s->stream), "upload");
      ck(cudaMemcpyAsync(in.p, selectors, sel_polys * pw * 8, cudaMemcpyHostToDevice, s->stream),
         "upload");
      opir::launch_split_u64(s->dp, in.p, s->sel.p, 1, sel_polys, 0, s->stream);
    }
    const uint32_t *r = run_other_dims(s, 1);
    DevBuf<uint64_t> o;
    o.alloc(2 * pw);
    opir::launch_compose_u64(s->dp, r, 0, o.p, 1, 2, s->stream);
    ck(cudaMemcpyAsync(out, o.p, 2 * pw * 8, cudaMemcpyDeviceToHost, s->stream), "download");
    ck(cudaStreamSynchronize(s->stream), "evaluate_other_dim");
  });
}

opir_status opir_server_ext_prod_mux(opir_server *s, const uint64_t *x, const uint64_t *y,
                                     const uint64_t *selector, uint64_t *out) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (!x || !y || !selector || !out) throw std::invalid_argument("null argument");
    DeviceGuard g(s->device);
    if (s->c4) return s->c4->ext_prod_mux(x, y, selector, out);
    // one MUX level of a two-candidate tree: level 0 pairs candidates 0, 1
    opir::Shape sh = s->shape;
    sh.other = 2;
    sh.num_dims = 2;
    const uint64_t sel_polys = 2ull * 2 * sh.l_ep;
    const uint64_t pw = poly_words(s->params);
    check_query_values(s, x, 2 * pw);
    check_query_values(s, y, 2 * pw);
    check_query_values(s, selector, sel_polys * pw);
    DevBuf<uint64_t> in;
    DevBuf<uint32_t> xy, res, sel;
    in.alloc(std::max<uint64_t>(4, sel_polys) * pw);
    xy.alloc(2 * kCtWords);
    res.alloc(2 * kCtWords);
    sel.alloc(sel_polys / 2 * kCtWords);
    ck(cudaMemcpyAsync(in.p, x, 2 * pw * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    ck(cudaMemcpyAsync(in.p + 2 * pw, y, 2 * pw * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    opir::launch_split_u64(s->dp, in.p, xy.p, 1, 4, 0, s->stream);
    ck(cudaStreamSynchronize(s->stream), "upload");
    ck(cudaMemcpyAsync(in.p, selector, sel_polys * pw * 8, cudaMemcpyHostToDevice, s->stream),
       "upload");
    opir::launch_split_u64(s->dp, in.p, sel.p, 1, sel_polys, 0, s->stream);
    opir::launch_mux_level(s->dp, sh, 0, 1, xy.p, res.p, 2, sel.p, 1, s->stream);
    opir::launch_compose_u64(s->dp, res.p, 0, in.p, 1, 2, s->stream);
    ck(cudaMemcpyAsync(out, in.p, 2 * pw * 8, cudaMemcpyDeviceToHost, s->stream), "download");
    ck(cudaStreamSynchronize(s->stream), "ext_prod_mux");
  });
}

opir_status opir_params_query_shape(const opir_params *scheme, const opir_query_shape *shape,
                                    opir_params *out) {
  if (!scheme || !shape || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] { *out = opir::with_query_shape(*scheme, *shape); });
}

opir_status opir_tree_params_make(uint64_t L, uint64_t a, uint64_t n, uint64_t ell_beta,
                                  uint64_t ell_gamma, uint64_t t, const uint64_t *moduli,
                                  uint32_t n_moduli, opir_tree_params *out) {
  if (!out || (n_moduli && !moduli)) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    *out = opir::make_tree_params(L, a, n, ell_beta, ell_gamma, t,
                                  std::vector<uint64_t>(moduli, moduli + n_moduli));
  });
}

opir_status opir_tree_params_init(uint64_t L, uint64_t a, const opir_params *scheme,
                                  opir_tree_params *out) {
  if (!scheme || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] { *out = opir::tree_params_for_scheme(L, a, *scheme); });
}

opir_status opir_tree_level_plans(const opir_tree_params *tree, opir_tree_level_plan *out) {
  if (!tree || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    const auto plans = opir::level_plans(*tree);
    std::copy(plans.begin(), plans.end(), out);
  });
}

opir_status opir_tree_query_params(const opir_tree_params *tree, const opir_params *scheme,
                                   opir_params *out) {
  if (!tree || !scheme || !out) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    opir::validate_tree_params(*tree, opir::scheme_moduli(*scheme));
    *out = opir::with_query_shape(
        *scheme, opir_query_shape{tree->N0, static_cast<uint32_t>(tree->b + tree->r),
                                  static_cast<uint32_t>(tree->h_q)});
  });
}

opir_status opir_tree_level_create(const opir_params *scheme, const opir_tree_params *tree,
                                   uint64_t level, const uint64_t *plaintexts, int device,
                                   opir_server **out) {
  if (!scheme || !tree || !plaintexts || !out) return OPIR_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  opir_params mp{};
  opir::LevelMatrix m;
  opir_tree_level_plan plan{};
  const opir_status vs = guarded(nullptr, [&] {
    const opir_params sch = checked_params(*scheme);
    if (is_k2mp(sch) || is_k1p(sch))
      throw std::invalid_argument("tree PIR is built for CONFIG_N2048_K1_COMP and CONFIG_N4096_K2_MP");
    const auto mods = opir::scheme_moduli(sch);
    opir::validate_tree_params(*tree, mods);
    if (tree->n != sch.poly_degree || tree->t != sch.plain_mod || tree->ell_beta != sch.l_ep ||
        tree->ell_gamma != sch.l_ep)
      throw std::invalid_argument("tree parameters are not bound to this scheme");
    if (level > tree->L) throw std::invalid_argument("tree_select: level is out of range");
    plan = opir::level_plans(*tree)[level];
    for (uint64_t i = 0; i < plan.R * tree->n; ++i)
      if (plaintexts[i] >= tree->t)
        throw std::invalid_argument("tree level coefficient exceeds the plaintext modulus");
    m = opir::arrange_level(*tree, plan, plaintexts);
    // the level as a rows x N0 first dimension followed by `fold` MUX steps
    // (levels 1..fold of a tree of height fold + 1), no expansion
    mp = sch;
    mp.fst_dim_sz = m.cols;
    mp.other_dim_sz = m.rows;
    mp.num_pt = mp.target_num_pt = m.rows * m.cols;
    mp.num_dims = static_cast<uint32_t>(m.fold + 2);
    mp.expansion_height = 0;
    mp.fst_dim_pow2 = 1;
    mp.view = OPIR_VIEW_MATRIX;
  });
  if (vs != OPIR_OK) return vs;
  opir_server *s = nullptr;
  const opir_status cs = create_handle(mp, device, &s);
  if (cs != OPIR_OK) return cs;
  const opir_status ls = guarded(s, [&] {
    s->tree_b = tree->b;
    s->fold_begin = plan.beta_begin;
    s->fold_count = plan.beta_count;
    DeviceGuard g(s->device);
    const uint64_t npt = m.rows * m.cols;
    if (s->c4) return s->c4->load_db(npt, m.coeffs.data());
    load_tiles(s, npt, [&](uint64_t b, uint64_t e, uint16_t *dst) {
      for (uint64_t i = 0; i < (e - b) * kN; ++i) dst[i] = static_cast<uint16_t>(m.coeffs[b * kN + i]);
    });
  });
  if (ls != OPIR_OK) {
    opir_server_destroy(s);
    return ls;
  }
  *out = s;
  return OPIR_OK;
}

opir_status opir_tree_select_level(opir_server *s, const uint64_t *alpha,
                                   const uint64_t *beta_selectors, uint64_t *out) {
  if (!s) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(s, [&] {
    if (s->params.view != OPIR_VIEW_MATRIX)
      throw std::invalid_argument("opir_tree_select_level needs a tree level handle");
    if (!alpha || !out || (s->fold_count && !beta_selectors))
      throw std::invalid_argument("null argument");
    const uint32_t fold = static_cast<uint32_t>(s->fold_count);
    const bool c4 = s->c4 != nullptr;
    const size_t ct_words = (c4 ? 4ull : 2ull) * s->params.poly_degree;
    const size_t sel_words = 2ull * s->params.l_ep * ct_words;
    // fold_beta_dimension (src/tree_select.cpp:175-201): step k consumes beta
    // bit begin + count - 1 - k (MSB first)
    std::vector<uint64_t> fold_sel(static_cast<size_t>(fold) * sel_words);
    for (uint32_t k = 0; k < fold; ++k) {
      const uint64_t u = s->fold_begin + s->fold_count - 1 - k;
      if (u >= s->tree_b) throw std::invalid_argument("fold needs a selector for every active beta bit");
      std::copy(beta_selectors + u * sel_words, beta_selectors + (u + 1) * sel_words,
                fold_sel.begin() + k * sel_words);
    }
    DeviceGuard g(s->device);
    if (c4) return s->c4->select_fold(alpha, fold_sel.data(), fold, out);
    const uint64_t q = s->params.q;
    for (size_t i = 0; i < s->shape.n0 * ct_words; ++i)
      if (alpha[i] >= q) throw std::invalid_argument("ciphertext coefficient not reduced mod q");
    for (uint64_t v : fold_sel)
      if (v >= q) throw std::invalid_argument("selector value not reduced mod q");
    select_fold_k1(s, alpha, fold_sel.data(), fold, out);
  });
}

void opir_tree_destroy(opir_tree *t) {
  if (!t) return;
  {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(t->device);
    if (t->stream) cudaStreamSynchronize(t->stream);
    for (opir_server *l : t->levels) opir_server_destroy(l);
    if (t->q) opir_server_destroy(t->q);
    for (cudaEvent_t e : t->done) cudaEventDestroy(e);
    if (t->q_done) cudaEventDestroy(t->q_done);
    t->out.reset();
    if (t->stream) cudaStreamDestroy(t->stream);
    if (prev >= 0) cudaSetDevice(prev);
  }
  delete t;
}

const char *opir_tree_last_error(const opir_tree *t) {
  return t ? t->last_error.c_str() : "null tree handle";
}

opir_status opir_tree_create(const opir_params *scheme, const opir_tree_params *tree,
                             const uint64_t *const *level_plaintexts, int device,
                             opir_tree **out) {
  if (!scheme || !tree || !level_plaintexts || !out) return OPIR_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  opir_tree *t = new (std::nothrow) opir_tree();
  if (!t) return OPIR_ERR_NO_MEMORY;
  const opir_status st = guarded_to(&t->last_error, [&] {
    t->tree = *tree;
    t->device = device;
    opir_params qp{};
    if (opir_tree_query_params(tree, scheme, &qp) != OPIR_OK)
      throw std::invalid_argument("tree parameters do not fit the scheme");
    if (create_handle(checked_params(qp), device, &t->q) != OPIR_OK)
      throw std::runtime_error("tree query handle could not be created");
    for (uint64_t l = 0; l <= tree->L; ++l) {
      if (!level_plaintexts[l]) throw std::invalid_argument("null level plaintexts");
      opir_server *h = nullptr;
      const opir_status ls = opir_tree_level_create(scheme, tree, l, level_plaintexts[l], device, &h);
      if (ls != OPIR_OK)
        throw std::runtime_error("tree level " + std::to_string(l) + " could not be created (status " +
                                 std::to_string(ls) + ")");
      t->levels.push_back(h);
    }
    DeviceGuard g(device);
    ck(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&t->q_done, cudaEventDisableTiming), "event");
    t->done.resize(t->levels.size(), nullptr);
    for (auto &e : t->done) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    // no allocation while answering
    if (t->q->c4) {
      t->out.alloc((tree->L + 1) * 4ull * scheme->poly_degree);
      t->q->c4->reserve(1);
      for (opir_server *l : t->levels) l->c4->reserve(1);
    } else {
      t->out.alloc((tree->L + 1) * 2ull * kN);
      ensure_capacity(t->q, 1);
      grow_keyptr_slots(t->q, 2);
      for (opir_server *l : t->levels) ensure_capacity(l, 1);
    }
  });
  if (st != OPIR_OK) {
    opir_tree_destroy(t);
    return st;
  }
  *out = t;
  return OPIR_OK;
}

opir_status opir_tree_set_client_keys(opir_tree *t, uint64_t client_id, const uint64_t *bv_keys,
                                      const uint32_t *galois_ks, uint32_t n_keys,
                                      const uint64_t *gsw_key) {
  if (!t) return OPIR_ERR_INVALID_ARGUMENT;
  const opir_status st = opir_server_set_client_keys(t->q, client_id, bv_keys, galois_ks, n_keys, gsw_key);
  t->last_error = t->q->last_error;
  return st;
}

opir_status opir_tree_query(opir_tree *t, uint64_t client_id, const uint64_t *query,
                            uint64_t *selected) {
  if (!t) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded_to(&t->last_error, [&] {
    if (!query || !selected) throw std::invalid_argument("null argument");
    opir_server *q = t->q;
    DeviceGuard g(t->device);
    if (q->c4) {  // two-limb set: the same flow through opir4::Server
      const size_t ct = 4ull * q->params.poly_degree;
      q->c4->tree_unpack(client_id, query);
      ck(cudaEventRecord(t->q_done, q->stream), "event record");
      for (size_t l = 0; l < t->levels.size(); ++l) {
        opir_server *ls = t->levels[l];
        ck(cudaStreamWaitEvent(ls->stream, t->q_done, 0), "wait");
        ls->c4->tree_select_device(q->c4->tree_leaves(), q->c4->tree_selectors(), ls->fold_begin,
                                   ls->fold_count, t->out.p + l * ct);
        ck(cudaEventRecord(t->done[l], ls->stream), "event record");
        ck(cudaStreamWaitEvent(t->stream, t->done[l], 0), "wait");
      }
      ck(cudaMemcpyAsync(selected, t->out.p, t->levels.size() * ct * 8, cudaMemcpyDeviceToHost,
                         t->stream), "download");
      ck(cudaStreamSynchronize(t->stream), "tree query");
      for (opir_server *ls : t->levels) ls->c4->check_device_error();
      return;
    }
    check_query_values(q, query, 2 * kN);
    // unpack_tree_query (src/tree_query.cpp:198-240) on the query handle
    ensure_capacity(q, 1);
    upload_keyptrs(q, &client_id, 1);
    ck(cudaMemcpyAsync(q->q_u64.p, query, 2 * kN * 8, cudaMemcpyHostToDevice, q->stream), "upload");
    opir::launch_split_u64(q->dp, q->q_u64.p, q->lvl[0].p, 1, 2, q->lvl_slots * kCtWords, q->stream);
    const uint32_t *leaves = run_expand(q, 1);
    opir::launch_selectors(q->dp, q->shape, leaves, q->lvl_slots, q->keyptrs.p + 1, q->sel.p, 1,
                           q->stream);
    ck(cudaEventRecord(t->q_done, q->stream), "event record");
    // select_level of every level on its own stream, inputs device to device
    const uint64_t sel_words = 2ull * q->params.l_ep * kCtWords;  // u32 words per selector
    for (size_t l = 0; l < t->levels.size(); ++l) {
      opir_server *ls = t->levels[l];
      ck(cudaStreamWaitEvent(ls->stream, t->q_done, 0), "wait");
      ck(cudaMemcpyAsync(ls->lvl[0].p, leaves, ls->shape.n0 * kCtWords * 4,
                         cudaMemcpyDeviceToDevice, ls->stream), "alpha copy");
      run_first_dim(ls, ls->lvl[0].p, 1);
      const uint32_t fold = static_cast<uint32_t>(ls->fold_count);
      for (uint32_t a = 1; a <= fold; ++a) {  // MSB-first: step a takes beta bit begin+count-a
        const uint64_t u = ls->fold_begin + ls->fold_count - a;
        ck(cudaMemcpyAsync(ls->sel.p + a * sel_words, q->sel.p + u * sel_words, sel_words * 4,
                           cudaMemcpyDeviceToDevice, ls->stream), "selector copy");
      }
      for (uint32_t a = 1; a <= fold; ++a)
        opir::launch_mux_level(ls->dp, ls->shape, a, ls->shape.num_dims - 1,
                               ls->mid[(a - 1) & 1].p, ls->mid[a & 1].p, ls->shape.other,
                               ls->sel.p, 1, ls->stream);
      const uint32_t *res = fold ? ls->mid[fold & 1].p : ls->mid[0].p;
      opir::launch_compose_u64(ls->dp, res, 0, t->out.p + l * 2ull * kN, 1, 2, ls->stream);
      ck(cudaEventRecord(t->done[l], ls->stream), "event record");
      ck(cudaStreamWaitEvent(t->stream, t->done[l], 0), "wait");
    }
    ck(cudaMemcpyAsync(selected, t->out.p, t->levels.size() * 2ull * kN * 8, cudaMemcpyDeviceToHost,
                       t->stream), "download");
    ck(cudaStreamSynchronize(t->stream), "tree query");
    for (opir_server *ls : t->levels) check_device_error(ls);
  });
}

opir_status opir_measure_butterfly_rate(opir_config config, int device, double *per_s) {
  // CONFIG_N2048_K2_MP runs on the residue-pair NTT of CONFIG_N2048_K1_COMP;
  // CONFIG_N2048_K1 on 64-bit Shoup butterflies like CONFIG_N4096_K2_MP
  if (!per_s || (config != OPIR_CONFIG_N2048_K1_COMP && config != OPIR_CONFIG_N4096_K2_MP &&
                 config != OPIR_CONFIG_N2048_K2_MP && config != OPIR_CONFIG_N2048_K1))
    return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    int sms = 0;
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    const bool c4 = config == OPIR_CONFIG_N4096_K2_MP || config == OPIR_CONFIG_N2048_K1;
    const uint32_t blocks = c4 ? opir4::bfly_rate_blocks(sms) : opir::bfly_rate_blocks(sms);
    const uint32_t iters = c4 ? 256 : 1024;
    *per_s = probe_rate(device, static_cast<size_t>(blocks) * 256, [&](uint64_t *sink, cudaStream_t st) {
      return c4 ? opir4::launch_bfly_rate(sink, blocks, iters, st)
                : opir::launch_bfly_rate(reinterpret_cast<uint32_t *>(sink), blocks, iters, st);
    });
  });
}

opir_status opir_measure_recombine_rate(int classes, int device, double *per_s) {
  if (!per_s || (classes != 5 && classes != 7)) return OPIR_ERR_INVALID_ARGUMENT;
  return guarded(nullptr, [&] {
    int sms = 0;
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "sm count");
    const uint32_t blocks = opir::recombine_rate_blocks(sms, classes);
    *per_s = probe_rate(device, static_cast<size_t>(blocks) * 128, [&](uint64_t *sink, cudaStream_t st) {
      return opir::launch_recombine_rate(reinterpret_cast<uint32_t *>(sink), blocks, 512, classes, st);
    });
  });
}

size_t opir_save_response(const opir_params *params, const uint64_t *resp, uint8_t *out,
                          size_t cap) {
  if (!params || !resp || !out) return 0;
  const uint32_t w = params->small_q_width;
  const size_t need = resp_bytes_of(*params);
  if (cap < need) return 0;
  uint8_t buf = 0;
  uint32_t filled = 0;
  size_t nb = 0;
  for (uint32_t i = 0; i < 2 * params->poly_degree; ++i) {
    const uint64_t c = resp[i] & ((1ull << w) - 1);
    uint32_t written = 0;
    while (written < w) {
      const uint32_t room = 8 - filled;
      const uint32_t take = std::min(room, w - written);
      buf |= static_cast<uint8_t>(((c >> written) & ((1ull << take) - 1)) << filled);
      filled += take;
      written += take;
      if (filled == 8) { out[nb++] = buf; buf = 0; filled = 0; }
    }
  }
  if (filled) out[nb++] = buf;
  return nb;
}

}  // extern "C"
