// Server state and query pipeline for the parameter sets whose limbs are
// 64-bit words: CONFIG_N4096_K2_MP (includes/database_constants.h:111-125,
// two 60-bit limbs at N = 4096) and CONFIG_N2048_K1 (:61-76, one 60-bit
// prime at N = 2048; no row shards or tree levels). The C-ABI handle
// forwards to this class when it was created with either set; argument
// checking that does not depend on the parameter set stays in the C-ABI
// layer. Ciphertexts are [c0][c1] with each polynomial limb-major (2 N K
// u64).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <set>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/onionpir_b200.h"
#include "opir_c4_kernels.h"
#include "opir_host.h"
#include "opir_k1p_kernels.h"
#include "opir_shard.h"

namespace opir4 {

class Server {
 public:
  // Stage-boundary events of one timed call: kMarks events recorded at the
  // stage boundaries (0..5) and around the scan (6, 7); null = untimed.
  using Events = cudaEvent_t *;
  static constexpr int kMarks = 8;

  // rs: a row shard of the layout (opir_shard.h): the database holds the
  // shard's rows, make_query returns the shard's partial ciphertext (4N u64)
  // after MUX levels 0 .. rs->tree_h - 1, and combine_* finishes the tree.
  Server(const opir_params &p, cudaStream_t stream, const opir::RowShard *rs = nullptr);
  Server(const Server &) = delete;
  Server &operator=(const Server &) = delete;
  ~Server();

  const opir_params &params() const { return p_; }
  bool db_loaded() const { return db_loaded_; }

  // server.cpp:80-203; coefficients are host arrays (each < t)
  void load_db(uint64_t logical, const uint64_t *coeffs);
  void load_db_u16(uint64_t logical, const uint16_t *coeffs);
  void load_db_source(uint64_t logical, opir_plaintext_source source, void *user);
  void load_db_seeded(uint64_t logical, uint64_t seed);

  void set_client_keys(uint64_t id, const uint64_t *bv_keys, const uint32_t *galois_ks,
                       uint32_t n_keys, const uint64_t *gsw_key);
  void remove_client(uint64_t id);

  // Host buffers: n queries of 4N u64 in, n responses of 2N u64 out (row
  // shard: n partial ciphertexts of 4N u64).
  void make_query_batch(uint32_t n, const uint64_t *ids, const uint64_t *queries,
                        uint64_t *responses, Events ev);
  // Device buffers, enqueued on the handle's stream (no wait).
  void make_query_batch_device(uint32_t n, const uint64_t *ids, const uint64_t *d_queries,
                               uint64_t *d_responses, Events ev);
  void reserve(uint32_t max_batch);
  // The stream the handle's work is enqueued on from now on (the caller has
  // synchronised the previous one).
  void set_stream(cudaStream_t st) { st_ = st; }
  // Limit of each tensor-core scan pipeline wait in clock cycles (0: the
  // default, about one second); drops the captured pipelines that hold the
  // old limit.
  void set_scan_wait_limit(long long cycles) {
    if (cycles != scan_wait_) clear_graphs();
    scan_wait_ = cycles;
  }
  static void plan_memory(const opir_params &p, opir_memory_plan *out);

  // Public stages of make_query (host buffers, reference layouts).
  void expand_query(uint64_t id, const uint64_t *query, uint64_t *out);
  void complete_selectors(uint64_t id, const uint64_t *expanded, uint64_t *out);
  void evaluate_first_dim(const uint64_t *fst_query, uint64_t *out);
  void evaluate_other_dim(const uint64_t *mid, const uint64_t *selectors, uint64_t *out);
  // ext_prod_mux (server.cpp:652-722) of one pair, host buffers: x, y and
  // out 4N u64 coefficient form, sel 2 L_EP rows x 4N u64 NTT form.
  void ext_prod_mux(const uint64_t *x, const uint64_t *y, const uint64_t *sel, uint64_t *out);
  // Row shards: the last log2 G MUX levels over each query's G partial
  // ciphertexts (G x n x 4N u64, shard-major), with the selectors of this
  // handle's last batch, then the modulus switch (n x 2N u64 out).
  void combine_host(uint32_t n, const uint64_t *partials, uint64_t *responses);
  void combine_device(uint32_t n, const uint64_t *d_partials, uint64_t *d_responses);
  // Tree level handles: first dimension over the n0 ciphertexts, then `fold`
  // MUX steps at levels 1..fold (selector slot a = step a), host buffers.
  void select_fold(const uint64_t *alpha, const uint64_t *fold_sel, uint32_t fold, uint64_t *out);

  // Device-resident tree (opir_tree_query), on the handle's stream, after
  // reserve(1). Query-shape handle: unpack_tree_query of a host query into
  // the handle's leaves (tree_leaves(), n0 alpha ciphertexts first) and
  // selector rows (tree_selectors(), 2 L_EP rows of kRowWords per selector).
  void tree_unpack(uint64_t id, const uint64_t *query);
  const uint64_t *tree_leaves() const { return lvl_[sh_.h & 1].p; }
  const uint64_t *tree_selectors() const { return sel_.p; }
  // Level handle: select_level from the query handle's device leaves and
  // selectors (fold step a takes selector fold_begin + fold_count - a) into
  // d_out (one ciphertext, kCt u64).
  void tree_select_device(const uint64_t *d_leaves, const uint64_t *d_selectors,
                          uint64_t fold_begin, uint64_t fold_count, uint64_t *d_out);
  // Reads and clears the tensor-core scan's error word (stream must be idle).
  void check_device_error();

 private:
  struct Keys {
    opir::DevBuf<uint64_t> bv, gsw;
  };
  struct PtrSlot {
    const uint64_t **host = nullptr;
    size_t cap = 0;
    cudaEvent_t done = nullptr;
  };
  static constexpr int kPtrSlots = 4;

  void ensure_capacity(uint32_t n);
  void upload_keyptrs(const uint64_t *ids, uint32_t n);
  void grow_ptr_slots(size_t entries);
  void check_ct_values(const uint64_t *v, size_t cts) const;
  void stage_in(const uint64_t *d_queries, uint32_t n);
  const uint64_t *run_expand(uint32_t n, bool *ntt_first = nullptr);
  void run_first_dim(const uint64_t *leaves, uint32_t n, Events ev, bool leaves_ntt = false);
  const uint64_t *run_other_dims(uint32_t n);
  void run_pipeline(uint32_t n, const uint64_t *ids, const uint64_t *d_queries,
                    uint64_t *d_resp, Events ev);
  void enqueue_core(uint32_t n, const uint64_t *d_queries, uint64_t *d_resp, Events ev);
  void launch_graph(uint32_t n, Events ev);
  void clear_graphs();
  void mark(Events ev, int i);
  void launch_scan(const uint8_t *qb, uint64_t *cmat, uint32_t n);
  void setup_k1_tables();
  void setup_c4_tables();
  opir1::Dev1 d1() const;
  void run_db_preprocess(const uint64_t *coeffs, uint64_t coeff_pt_begin, uint64_t seed,
                         uint64_t logical, uint64_t pb, uint64_t pe);
  void run_selectors(const uint64_t *leaves, const uint64_t *const *gsw, uint32_t n);
  void run_mux(const Shape4 &sh, uint32_t level, uint32_t tree_h, const uint64_t *in, uint64_t *out,
               uint64_t mid_stride, const uint64_t *sel, uint32_t n);
  void run_modswitch(const uint64_t *ct, uint64_t ct_stride, uint64_t *resp, uint32_t n);
  template <typename Fill>
  void load_tiles(uint64_t logical, Fill &&fill);

  opir_params p_{};
  bool k1_ = false;          // CONFIG_N2048_K1 (opir_k1p_kernels.h) instead of CONFIG_N4096_K2_MP
  uint32_t n_ = kN;          // ring degree N
  uint32_t limbs_ = 2;       // RNS limbs K
  uint64_t ct_ = kCtWords;   // u64 words per ciphertext: 2 N K
  uint64_t row_ = kRowWords; // u64 words per key / selector row: ciphertext + companions
  Shape4 sh_{};
  Dev4 dp_{};
  cudaStream_t st_ = nullptr;
  opir::DevBuf<ulonglong2> tables_;
  opir::DevBuf<uint8_t> db8_;   // byte-plane database (opir_c4_kernels.h)
  CUtensorMap map_db_{};        // TMA view of db8_ for the tensor-core scan
  opir::DevBuf<uint32_t> err_;  // error word of the tensor-core scan
  opir::DevBuf<uint32_t> progress_;  // scan CTA pairing counters
  int sm_count_ = 148;
  long long scan_wait_ = 0;     // scan pipeline wait limit (0: default)
  bool db_loaded_ = false;
  // MUX levels answered here; on a row shard the rows kept (local -> database)
  uint32_t tree_h_ = 0, num_shards_ = 1;
  std::vector<uint32_t> host_rows_;
  opir::DevBuf<uint32_t> row_map_;
  opir::DevBuf<uint64_t> comb_[2];
  uint64_t out_words_ = 2ull * kN;  // per query out of make_query: 2N, or a ciphertext on a shard
  bool shard_ = false;              // a row shard (opir_shard.h) of the layout
  std::unordered_map<uint64_t, Keys> clients_;
  uint32_t cap_ = 0;
  uint64_t lvl_slots_ = 1;
  opir::DevBuf<uint64_t> q_in_, resp_, lvl_[2], sel_, mid_[2];
  opir::DevBuf<const uint64_t *> keyptrs_;
  std::vector<const uint64_t *> host_ptrs_;
  PtrSlot ring_[kPtrSlots];
  uint32_t ring_next_ = 0;
  // captured pipelines per (batch size, timed): eager on first use, captured
  // on the second; ev_nodes[i] = event-record node of stage mark i
  struct Graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    std::vector<cudaGraphNode_t> ev_nodes;
  };
  bool use_graphs_ = true;
  std::map<std::tuple<uint32_t, bool>, Graph> graphs_;
  std::set<std::tuple<uint32_t, bool>> graph_seen_;
};

// Parameters of the two-limb set for a layout (pir.cpp:49-134).
opir_params derive(const opir_layout &layout);

}  // namespace opir4
