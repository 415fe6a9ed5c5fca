/* onionpir_b200.h -- C ABI of the B200 OnionPIRv2 server hot path.
 *
 * This library replaces the reference's PirServer query-processing path
 * (src/server.cpp, src/gsw.cpp, src/bv_keyswitch.cpp, src/matrix.cpp of
 * zcy05331/OnionPIRv2) with hand-written sm_100a CUDA kernels. Every entry
 * point below names the reference interface it replaces (paths relative to
 * the reference's src/). Two parameter sets (includes/database_constants.h):
 *   CONFIG_N2048_K1_COMP (:77-94): N = 2048, logical q = q1*q2 with two
 *     29-bit NTT primes, t = 4099, small_q = 4169729, L_EP = 6, L_KEY = 10,
 *     L_KS = 8 (opir_params_init);
 *   CONFIG_N4096_K2_MP (:111-125): N = 4096, two 60-bit RNS limbs
 *     q0 = 1152921504606830593, q1 = 1152921504606748673, t =
 *     generate_prime(40), 50-bit small_q, L_EP = 5, L_KEY = 8, L_KS = 8
 *     (opir_params_init_config).
 *
 * Conventions
 *   - Plain pointers and sizes only. Host buffers unless a name ends in
 *     _device, in which case the pointers are CUDA device pointers.
 *   - Every call returns an opir_status (0 = OK). A non-zero status never
 *     leaves a CUDA error pending; opir_server_last_error() describes it. The
 *     status codes map onto the exception types the reference throws.
 *   - Ciphertexts are [c0 (N u64)][c1 (N u64)], coefficients canonical in
 *     [0, q) (includes/rlwe.h:17-31, K = 1). Key rows are in the NTT domain of
 *     the reference's NTT (HEXL ordering: forward output bit-reversed,
 *     root = CRT of the minimal primitive 2N-th roots mod q1 and q2).
 *     Under CONFIG_N4096_K2_MP every polynomial is limb-major,
 *     [limb 0 (N)][limb 1 (N)], so a ciphertext is 4N u64, each limb
 *     canonical mod its prime and NTT rows per limb (root = the minimal
 *     primitive 2N-th root of that limb); the sizes quoted below in N double
 *     accordingly (2N -> 4N per ciphertext, N -> 2N per key polynomial).
 *   - A server handle owns its device memory (database, client keys, scratch
 *     arena) on the device it was created on. Calls on one handle must not
 *     run concurrently; distinct handles are independent.
 */
#ifndef ONIONPIR_B200_H
#define ONIONPIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  OPIR_OK = 0,
  OPIR_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
  OPIR_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range (unknown client, index) */
  OPIR_ERR_RUNTIME = 3,          /* std::runtime_error */
  OPIR_ERR_CUDA = 4,             /* CUDA launch/runtime failure */
  OPIR_ERR_NO_MEMORY = 5,        /* device allocation failed / HBM budget */
  OPIR_ERR_OVERFLOW = 6          /* std::overflow_error */
} opir_status;

/* ACTIVE_CONFIG choices (includes/database_constants.h:31-40) that this
 * library implements. */
typedef enum {
  OPIR_CONFIG_N2048_K1_COMP = 0,
  OPIR_CONFIG_N4096_K2_MP = 1,
  OPIR_CONFIG_N2048_K2_MP = 2,
  OPIR_CONFIG_N2048_K1 = 3
} opir_config;

/* PirLayoutConfig (includes/pir.h:199-203). */
typedef struct {
  uint64_t target_num_pt;
  uint32_t expansion_height;
  uint32_t fst_dim_pow2;
} opir_layout;

/* Derived runtime parameters: the values PirParams exposes through its
 * getters (includes/pir.h:237-277, src/pir.cpp:14-134). */
typedef struct {
  uint32_t poly_degree;           /* N */
  uint32_t num_limbs;             /* K (1: logical single modulus, 2: RNS) */
  uint64_t q;                     /* logical ciphertext modulus q1*q2 (K = 1,
                                     and K = 2 at N = 2048); 0 at N = 4096
                                     (the product needs 120 bits)          */
  uint64_t q1, q2;                /* composite first-dim limbs (K = 1), or the
                                     two RNS limbs (K = 2); 0 under
                                     CONFIG_N2048_K1 (q itself is prime)   */
  uint64_t w1, w2, w_crt;         /* 2N-th roots: q1, q2 and CRT (mod q) */
  uint64_t q1_inv_mod_q2;
  uint64_t plain_mod;             /* t                                   */
  uint64_t small_q;               /* modulus-switch target               */
  uint32_t small_q_width;         /* response bits per coefficient       */
  uint32_t ct_mod_width;          /* 58                                  */
  uint32_t l_ep, l_key, l_ks;     /* gadget lengths                      */
  uint32_t base_log2, base_log2_key, base_log2_ks;
  uint64_t target_num_pt, num_pt, fst_dim_sz, other_dim_sz;
  uint32_t num_dims, expansion_height, fst_dim_pow2;
  uint32_t view;                  /* opir_view: what a handle on these
                                     parameters may do (below)            */
} opir_params;

/* Views of a parameter set. OPIR_VIEW_LAYOUT: a database layout
 * (opir_params_init[_config]); every call is available. OPIR_VIEW_QUERY_SHAPE:
 * PirParams::with_query_shape (includes/pir.h:46-66) -- no database behind
 * it; a handle only expands queries and completes selectors
 * (opir_server_expand_query, opir_server_complete_selectors).
 * OPIR_VIEW_MATRIX: a tree PIR level database (opir_tree_level_create),
 * answered by opir_tree_select_level. OPIR_VIEW_ROW_SHARD: one GPU's rows
 * of a layout split across GPUs (opir_server_create_row_shard): loads and
 * the row-shard query calls. Calls outside a view's scope return
 * OPIR_ERR_INVALID_ARGUMENT. */
typedef enum {
  OPIR_VIEW_LAYOUT = 0,
  OPIR_VIEW_QUERY_SHAPE = 1,
  OPIR_VIEW_MATRIX = 2,
  OPIR_VIEW_ROW_SHARD = 3
} opir_view;

/* PirQueryShapeConfig (includes/pir.h:46-50). */
typedef struct {
  uint64_t fst_dim_sz;
  uint32_t num_selector_bits;
  uint32_t expansion_height;
} opir_query_shape;

typedef struct opir_server opir_server;

/* Plaintext source callback: fill out_coeffs[0..N) (each < t) for the given
 * logical plaintext index. Returns 0 on success. Replaces PlaintextSource
 * (includes/server.h:13). */
typedef int (*opir_plaintext_source)(void *user, uint64_t logical_index,
                                     uint64_t *out_coeffs);

/* ---- parameters ---------------------------------------------------------- */

/* PirParams().with_layout(layout) (src/pir.cpp:49-134). */
opir_status opir_params_init(const opir_layout *layout, opir_params *out);

/* PirParams under a chosen ACTIVE_CONFIG: CONFIG_N2048_K1_COMP gives the
 * same as opir_params_init, CONFIG_N4096_K2_MP the two-limb set
 * (src/pir.cpp:49-134 with RnsMods {60, 60}, PlainMod 40, SmallQWidth 50;
 * expansion_height <= 12), CONFIG_N2048_K2_MP the two-limb set at N = 2048
 * (RnsMods {29, 29} as real RNS limbs, PlainMod 10, SmallQWidth 22, L_EP 5,
 * L_KEY 8, L_KS 8, the MP gadgets; includes/database_constants.h:96-110;
 * expansion_height <= 11). Handles on CONFIG_N2048_K2_MP take ciphertexts,
 * keys and stage arrays limb-major (K = 2) like CONFIG_N4096_K2_MP and
 * answer make_query, its batch forms and the stage methods;
 * CONFIG_N2048_K1, the reference's default (includes/database_constants.h:
 * 61-76), one real 60-bit NTT prime at N = 2048 (num_limbs 1, q the prime,
 * q1 = q2 = 0), PlainMod 14, SmallQWidth 22, L_EP 5, L_KEY 8, L_KS 8 with
 * signed single-modulus digits (expansion_height <= 11), ciphertexts
 * [c0 (N)][c1 (N)] u64 mod q. Row shards and tree PIR are built for
 * CONFIG_N2048_K1_COMP and CONFIG_N4096_K2_MP. Unknown config ->
 * OPIR_ERR_INVALID_ARGUMENT. */
opir_status opir_params_init_config(opir_config config, const opir_layout *layout,
                                    opir_params *out);

/* PirParams::with_query_shape (src/pir.cpp:136-166): the scheme of `scheme`
 * with first dimension fst_dim_sz, 1 + num_selector_bits dimensions and the
 * given expansion height, num_pt = fst_dim_sz, view OPIR_VIEW_QUERY_SHAPE.
 * Shapes that do not fit the expansion capacity or exceed log2 N ->
 * OPIR_ERR_INVALID_ARGUMENT. */
opir_status opir_params_query_shape(const opir_params *scheme, const opir_query_shape *shape,
                                    opir_params *out);

/* Bytes of the serialized response: ceil(2 N small_q_width / 8). */
size_t opir_response_bytes(const opir_params *params);

/* ---- server lifetime ------------------------------------------------------ */

/* PirServer::PirServer(const PirParams&) (src/server.cpp:29-46). Allocates
 * the device database on CUDA device `device`. */
opir_status opir_server_create(const opir_params *params, int device,
                               opir_server **out);
/* PirServer::~PirServer (src/server.cpp:48-49). NULL is a no-op. */
void opir_server_destroy(opir_server *server);
/* Human-readable description of the last failure on this handle. */
const char *opir_server_last_error(const opir_server *server);
/* The parameters the server was created with. */
opir_status opir_server_params(const opir_server *server, opir_params *out);

/* ---- database ------------------------------------------------------------- */

/* PirServer::load_data (src/server.cpp:80-203) with the plaintexts given as
 * one host array: logical_num_pt x N coefficients, each < t. The rounded
 * tail [logical_num_pt, num_pt) is zero. NTT, CRT split and the transpose
 * into the coefficient-major first-dimension layout run on the device. */
opir_status opir_server_load_db(opir_server *server, uint64_t logical_num_pt,
                                const uint64_t *coeffs);
/* Same, 16-bit coefficients (t < 2^16), halving the host->device bytes. */
opir_status opir_server_load_db_u16(opir_server *server,
                                    uint64_t logical_num_pt,
                                    const uint16_t *coeffs);
/* Same, pulling plaintexts through a callback like the reference's
 * PlaintextSource; the callback is called once per logical index, in order. */
opir_status opir_server_load_db_source(opir_server *server,
                                       uint64_t logical_num_pt,
                                       opir_plaintext_source source,
                                       void *user);
/* Synthetic database generated on the device from a seed:
 * coefficient(pt, c) = mix64(seed + (pt*N + c + 1) * 0x9E3779B97F4A7C15) % t
 * (SplitMix64 finaliser). Used by benchmarks and tests. */
opir_status opir_server_load_db_seeded(opir_server *server,
                                       uint64_t logical_num_pt, uint64_t seed);

/* ---- client keys ---------------------------------------------------------- */

/* PirServer::set_client_bv_galois_key + set_client_gsw_key
 * (src/server.cpp:857-863) / set_client_session_keys (:865-875).
 *   bv_keys : n_keys x L_KS rows x [b (N)][a (N)] u64, NTT form
 *             (bvks::BvKeySwitchKey, includes/bv_keyswitch.h:48-66)
 *   galois_ks: n_keys automorphism exponents; every (N >> i) + 1 for
 *             i < expansion_height must be present
 *   gsw_key : 2 L_KEY rows x [c0 (N)][c1 (N)] u64, NTT form (GSWCt RGSW(s))
 * Re-registering a client id replaces its keys. */
opir_status opir_server_set_client_keys(opir_server *server, uint64_t client_id,
                                        const uint64_t *bv_keys,
                                        const uint32_t *galois_ks,
                                        uint32_t n_keys,
                                        const uint64_t *gsw_key);
/* Representation of the key rows handed to opir_server_set_client_keys_ex. */
typedef enum {
  OPIR_KEYS_NTT = 0,   /* this library's NTT domain (the Conventions above) */
  OPIR_KEYS_COEFF = 1  /* coefficient form */
} opir_key_form;

/* opir_server_set_client_keys with the rows' representation named. Key rows
 * made by a producer with another NTT convention (a client built on Intel
 * HEXL, whose NTT-domain order is its own) are handed over in coefficient
 * form -- the producer's own inverse NTT of each row, which no convention
 * affects -- as OPIR_KEYS_COEFF; the server takes every polynomial into its
 * NTT domain on the GPU and installs the keys as opir_server_set_client_keys
 * does. Same layouts, limbs and errors; a coefficient at or above its
 * limb's modulus is OPIR_ERR_INVALID_ARGUMENT. */
opir_status opir_server_set_client_keys_ex(opir_server *server, uint64_t client_id,
                                           const uint64_t *bv_keys,
                                           const uint32_t *galois_ks, uint32_t n_keys,
                                           const uint64_t *gsw_key, uint32_t key_form);
opir_status opir_server_remove_client(opir_server *server, uint64_t client_id);

/* ---- query processing ----------------------------------------------------- */

/* PirServer::make_query (src/server.cpp:895-947): expansion, selector
 * completion, first dimension, remaining dimensions, modulus switch.
 *   query    : [c0 (N)][c1 (N)] u64 coefficient form mod q
 *   response : [c0 (N)][c1 (N)] u64 coefficient form mod small_q
 * Unknown client_id -> OPIR_ERR_OUT_OF_RANGE (the reference's map::at). */
opir_status opir_server_make_query(opir_server *server, uint64_t client_id,
                                   const uint64_t *query, uint64_t *response);

/* Batched form: n independent queries (each with its own client) answered
 * in one pass, the first-dimension scan reading the database once for the
 * whole batch. queries: n x 2N u64; responses: n x 2N u64. */
opir_status opir_server_make_query_batch(opir_server *server, uint32_t n,
                                         const uint64_t *client_ids,
                                         const uint64_t *queries,
                                         uint64_t *responses);

/* Batched form on device-resident buffers, enqueued on `stream`
 * (a cudaStream_t; NULL = the handle's own stream). client_ids is a host
 * array. The call returns after enqueueing (it does not wait for earlier work
 * on the device; if the scratch arena must grow for n it allocates, see
 * opir_server_reserve); synchronise the stream before reading d_responses.
 * The next call on the same handle may be enqueued before this one has
 * finished: calls on one handle run in order on the handle's stream. */
opir_status opir_server_make_query_batch_device(opir_server *server, uint32_t n,
                                                const uint64_t *client_ids,
                                                const uint64_t *d_queries,
                                                uint64_t *d_responses,
                                                void *stream);

/* ---- row shards: one database across G GPUs ------------------------------
 * No counterpart in the reference (one PirServer holds the whole database).
 * A layout whose database exceeds one GPU is split by candidate rows over
 * G = 2^k GPUs (1 <= G <= 2^(num_dims-2)). evaluate_other_dim
 * (src/server.cpp:599-649) first pairs rows (level 0) into 2^(h-1)
 * positions s (h = num_dims - 1) and then halves along the top bit of s;
 * shard g holds the rows feeding the positions s with s mod G == g, so its
 * MUX levels 0 .. h-k-1 stay on the GPU and leave one ciphertext: the full
 * tree's level-(h-k) position g. The k remaining levels run on one shard
 * over the G gathered ciphertexts, followed by the modulus switch; the
 * response is bit for bit PirServer::make_query's.
 *
 * Rows of shard g in the order they are stored (database row indices;
 * rows may be NULL to query only the count) and the MUX levels it answers. */
opir_status opir_row_shard_rows(const opir_params *params, uint32_t shard,
                                uint32_t num_shards, uint32_t *rows,
                                uint64_t *n_rows, uint32_t *tree_h);
/* A handle holding shard `shard` of `num_shards` of a layout (params of view
 * OPIR_VIEW_LAYOUT; the handle reports view OPIR_VIEW_ROW_SHARD). Every load
 * call takes the whole database's arguments (logical count, the full host
 * array, or a source that is then called for the shard's plaintexts only,
 * in increasing index order) and keeps the shard's rows. */
opir_status opir_server_create_row_shard(const opir_params *params,
                                         uint32_t shard, uint32_t num_shards,
                                         int device, opir_server **out);
/* The shard's part of make_query for n queries: expansion and selectors
 * (replicated on every shard), the first dimension over the shard's rows and
 * its MUX levels. partials: n ciphertexts in the query layout
 * ([c0 K*N][c1 K*N] u64, coefficient form mod each limb). The handle keeps
 * the batch's selectors for opir_server_combine_shards. */
opir_status opir_server_make_query_shard_batch(opir_server *server, uint32_t n,
                                               const uint64_t *client_ids,
                                               const uint64_t *queries,
                                               uint64_t *partials);
/* Device-buffer form, enqueued like opir_server_make_query_batch_device. */
opir_status opir_server_make_query_shard_batch_device(opir_server *server,
                                                      uint32_t n,
                                                      const uint64_t *client_ids,
                                                      const uint64_t *d_queries,
                                                      uint64_t *d_partials,
                                                      void *stream);
/* Finishes n queries on a shard whose last make_query_shard batch had the
 * same client ids in the same order (else OPIR_ERR_INVALID_ARGUMENT):
 * partials = G x n ciphertexts, shard-major (shard g's batch output at
 * g * n), responses = n x 2N u64 mod small_q, as opir_server_make_query. */
opir_status opir_server_combine_shards(opir_server *server, uint32_t n,
                                       const uint64_t *client_ids,
                                       const uint64_t *partials,
                                       uint64_t *responses);
opir_status opir_server_combine_shards_device(opir_server *server, uint32_t n,
                                              const uint64_t *client_ids,
                                              const uint64_t *d_partials,
                                              uint64_t *d_responses,
                                              void *stream);

/* ---- device memory planning ---------------------------------------------
 * No counterpart in the reference (its server grows host vectors as it
 * goes). The device bytes a handle requests from the CUDA allocator (which
 * rounds each allocation up to its page size), so that a request loop can
 * admit databases, clients and in-flight batches against an HBM budget before
 * it allocates anything. Registering a client also holds a transient upload
 * buffer of max(BV, RGSW) key bytes / 2 for the duration of the call. */
typedef struct {
  uint64_t database_bytes;          /* byte-plane database, NTT tables, error word */
  uint64_t client_key_bytes;        /* one registered client's BV + RGSW keys */
  uint64_t scratch_bytes_per_query; /* scratch arena bytes per query of a batch */
  uint64_t scratch_bytes_fixed;     /* scratch arena bytes independent of the batch */
} opir_memory_plan;
opir_status opir_plan_memory(const opir_params *params, opir_memory_plan *out);

/* Grows the handle's scratch arena to max_batch queries now (a no-op when it
 * is already that large), so that later query calls with n <= max_batch
 * allocate no device memory and never wait on the CUDA allocator. The arena
 * then holds scratch_bytes_fixed + max_batch * scratch_bytes_per_query. */
opir_status opir_server_reserve(opir_server *server, uint32_t max_batch);

/* No counterpart in the reference (its matrix.cpp kernels have one fixed
 * blocking). Times the tilings of the tensor-core first-dimension scan --
 * query columns per tile (16, 32, 64), K bytes per pipeline stage (128 with
 * 128-byte swizzle, 64 with 64-byte swizzle) and pipeline depth -- on this
 * handle's database, and the cluster width of every expansion level (1, 2, 4
 * or 8 CTAs per key switch) and MUX level (1, 2 or, with an even digit
 * count, 4 CTAs per MUX), for batches of 1, 2, 4, ... up to max_batch
 * queries, and keeps the fastest per batch-size bucket. Every tiling and
 * width computes the same result; only the speed differs. Synchronises the
 * handle's stream and overwrites its scratch arena: no query may be in
 * flight on the handle. The residue-pair sets only (CONFIG_N2048_K1_COMP,
 * CONFIG_N2048_K2_MP); a no-op on the 64-bit-limb sets. */
opir_status opir_server_autotune(opir_server *server, uint32_t max_batch);
/* The scan tiling a batch of n queries uses (autotuned, else the default). */
opir_status opir_server_scan_tile(const opir_server *server, uint32_t n,
                                  uint32_t *ntile, uint32_t *kt,
                                  uint32_t *stages);
/* No counterpart in the reference. The cluster widths a batch of n queries
 * uses: expand[d] for expansion level d (16 entries), mux[a] for MUX level a
 * (32 entries); 0 means the default rule (split while a level has fewer CTAs
 * than the GPU has slots), else the autotuned width. */
opir_status opir_server_level_splits(const opir_server *server, uint32_t n, uint8_t *expand,
                                     uint8_t *mux);

/* No counterpart in the reference. Moves the handle's work to a new CUDA
 * stream of the given priority (cudaStreamCreateWithPriority: lower numbers
 * are scheduled first; values outside the device's range are clamped), after
 * the work already on the old stream has finished. A serving loop gives
 * databases whose queries are cheap a higher priority than those whose
 * batches hold the GPU for long, so cheap queries are not queued behind
 * expensive ones. Results do not depend on the priority. */
opir_status opir_server_set_priority(opir_server *server, int priority);

/* No counterpart in the reference. Every wait inside the tensor-core
 * first-dimension scan (a pipeline stage filled by TMA, the MMAs of a tile,
 * the epilogue handing back its accumulators) gives up after a limit; the
 * kernel then records an error code, lets its own copies and MMAs finish,
 * frees its tensor memory and returns, and the call fails with
 * OPIR_ERR_RUNTIME ("tensor-core scan timed out"). The default limit, about
 * one second of clock cycles, is far above any legitimate wait. This call
 * sets the limit in SM clock cycles (0 restores the default; at most 2^40),
 * so a test can make a wait run out and check that the handle reports it
 * and answers correctly afterwards. Waits while the kernel drains are not
 * affected. Synchronises the handle's stream. */
opir_status opir_server_set_scan_wait_limit(opir_server *server, uint64_t cycles);

/* Per-stage device times (ms), averaged over the make_query / batch calls
 * made since stage timing was (re-)enabled, in the reference's TimerLogger
 * sections (includes/logging.h:34-78): [0] Expand, [1] Convert,
 * [2] First dim, [3] Other dim, [4] Modulus switching, [5] Core (the
 * first-dimension scan kernel alone, the reference's CORE_TIME). Timing uses
 * CUDA events on the handle's stream; opir_server_stage_times synchronises
 * that stream. *calls receives the number of calls averaged (may be NULL). */
opir_status opir_server_set_stage_timing(opir_server *server, int enabled);
opir_status opir_server_stage_times(opir_server *server, float *ms_out,
                                    uint32_t *calls);

/* No counterpart in the reference. The rate (butterflies per second) at
 * which the device retires the NTT's forward radix-2 butterflies of the
 * parameter set -- the radix-8 register pass of the NTT kernels, with their
 * lazy-correction pattern, on register-resident values and twiddles, one
 * modular (Shoup) product each -- over every SM at full occupancy: the
 * denominator of the NTT-bound stages' roofline. Runs about a millisecond
 * of probe kernels on `device`. */
opir_status opir_measure_butterfly_rate(opir_config config, int device, double *per_s);

/* No counterpart in the reference. The rate (outputs per second) at which
 * the device finishes one output of an int8 tensor-core product of
 * byte-sliced 29-bit residues: `classes` (5 or 7) int32 shift-class sums
 * S_s combined as sum_s S_s (2^(8s) mod q) in 64 bits and Barrett-reduced
 * mod q -- the first-dimension scan's epilogue arithmetic -- on
 * register-resident sums over every SM, without the accumulator loads and
 * stores. A byte-sliced tensor-core NTT pays this once per coefficient per
 * matrix step, so the rate bounds such an NTT from above whatever the MMA
 * speed. Runs about a millisecond of probe kernels on `device`. */
opir_status opir_measure_recombine_rate(int classes, int device, double *per_s);

/* Total kernel launches issued by this library in this process. */
uint64_t opir_launch_count(void);

/* ---- individual stages (public PirServer methods used by tests and by the
 *      reference's tree-PIR callers) --------------------------------------- */

/* PirServer::expand_query (src/server.cpp:818-821): useful leaves
 * u = fst_dim_sz + L_EP (num_dims - 1), out: u x 2N u64 coefficient form. */
opir_status opir_server_expand_query(opir_server *server, uint64_t client_id,
                                     const uint64_t *query, uint64_t *out);
/* PirServer::complete_selectors (src/server.cpp:823-855): expanded is the
 * expand_query output; out: (num_dims-1) x 2 L_EP rows x 2N u64, NTT form. */
opir_status opir_server_complete_selectors(opir_server *server,
                                           uint64_t client_id,
                                           const uint64_t *expanded,
                                           uint64_t *out);
/* PirServer::evaluate_first_dim (src/server.cpp:313-405): fst_query is
 * fst_dim_sz x 2N u64 coefficient form; out: other_dim_sz x 2N u64
 * coefficient form. */
opir_status opir_server_evaluate_first_dim(opir_server *server,
                                           const uint64_t *fst_query,
                                           uint64_t *out);
/* PirServer::evaluate_other_dim (src/server.cpp:599-649): mid is
 * other_dim_sz x 2N coefficient form, selectors as produced by
 * complete_selectors; out: 2N u64 (before the modulus switch). */
opir_status opir_server_evaluate_other_dim(opir_server *server,
                                           const uint64_t *mid,
                                           const uint64_t *selectors,
                                           uint64_t *out);

/* PirServer::ext_prod_mux (src/server.cpp:652-722): out = x + b (y - x)
 * for the RGSW selector bit b. x, y, out: one ciphertext each in the query
 * layout, coefficient form; selector: 2 L_EP rows in the complete_selectors
 * layout (NTT form). Unlike the reference, y is not overwritten. Available
 * on every handle (it does not read the database). */
opir_status opir_server_ext_prod_mux(opir_server *server, const uint64_t *x,
                                     const uint64_t *y, const uint64_t *selector,
                                     uint64_t *out);

/* ---- response codec ------------------------------------------------------- */

/* PirServer::save_resp_to_stream (src/server.cpp:950-1009): c0 then c1,
 * small_q_width bits per coefficient, LSB-first, zero-padded last byte.
 * Returns the byte count, or 0 if cap is too small. Host-only helper (the
 * device path writes the same bytes in its modulus-switch kernel). */
size_t opir_save_response(const opir_params *params, const uint64_t *response,
                          uint8_t *out, size_t cap);

/* ---- wire codec: seed-compressed queries and client keys -----------------
 * No serializer exists in the reference; its communication model
 * (includes/pir.h:115-139) counts a 32-byte seed in place of every uniformly
 * random polynomial. This codec is that model as a format. Each uniform
 * polynomial -- a query's c1, the a of every BV key row, the c1 of every RGSW
 * row -- is Expand(seed, domain, index): the ChaCha20 block function
 * (RFC 8439) keyed by the seed, nonce = domain (u32 little-endian) || index
 * (u64 little-endian), block counter from 0, read as little-endian u64
 * words; limb k takes, coefficient by coefficient, the next word whose low
 * bit_length(q_k) bits are below q_k (limb-major; under
 * CONFIG_N2048_K1_COMP the one limb is the logical q). A client builds its
 * ciphertexts around these polynomials (opir_prf_expand): for an RGSW row
 * whose message sits in c1, it takes c1 from the seed and derives its `a`
 * as c1 - m g. The other polynomial is packed at bit_length(q_k) bits per
 * coefficient, LSB first, limb by limb.
 *   query   : "OPQ1" | seed | c0                      (k1_comp: 14,884 bytes)
 *   keys    : "OPK1" | seed | b of the h x L_KS BV rows (level-major, the
 *             galois_k of level i is (N >> i) + 1) | c0 of the 2 L_KEY RGSW
 *             rows                                  (k1_comp, h = 10: 1.49 MB)
 * Query indices: domain OPIR_PRF_QUERY, index 0; BV row j of level i:
 * OPIR_PRF_BV_KEY, index i L_KS + j; RGSW row r: OPIR_PRF_GSW_KEY, index r.
 * Encoders reject a uniform polynomial that is not Expand(seed) and any
 * unreduced coefficient (OPIR_ERR_INVALID_ARGUMENT); decoders reject a wrong
 * magic or length. */
#define OPIR_SEED_BYTES 32
typedef enum {
  OPIR_PRF_QUERY = 1,
  OPIR_PRF_BV_KEY = 2,
  OPIR_PRF_GSW_KEY = 3
} opir_prf_domain;
/* Expand(seed, domain, index): K x N u64. */
opir_status opir_prf_expand(const opir_params *params, const uint8_t *seed, uint32_t domain,
                            uint64_t index, uint64_t *out);
size_t opir_query_wire_bytes(const opir_params *params);
size_t opir_keys_wire_bytes(const opir_params *params);
/* query: the [c0][c1] ciphertext (c1 = Expand(seed, OPIR_PRF_QUERY, 0));
 * out: opir_query_wire_bytes bytes (cap at least that). */
opir_status opir_query_encode(const opir_params *params, const uint8_t *seed,
                              const uint64_t *query, uint8_t *out, size_t cap);
opir_status opir_query_decode(const opir_params *params, const uint8_t *in, size_t len,
                              uint64_t *query);
/* bv_keys / gsw_key in the opir_server_set_client_keys layouts, h =
 * params->expansion_height levels in galois order (N >> i) + 1;
 * decode also fills galois_ks (h entries). */
opir_status opir_keys_encode(const opir_params *params, const uint8_t *seed,
                             const uint64_t *bv_keys, const uint64_t *gsw_key,
                             uint8_t *out, size_t cap);
opir_status opir_keys_decode(const opir_params *params, const uint8_t *in, size_t len,
                             uint64_t *bv_keys, uint32_t *galois_ks, uint64_t *gsw_key);

/* ---- allocation-free MUX ------------------------------------------------- */

/* No counterpart in the reference. For callers that cannot allocate device
 * memory when they run a MUX step (a host that pre-budgets and owns all
 * device memory, or a request loop that must not touch the CUDA allocator
 * because an allocation can synchronise the device): n independent MUX
 * steps out_i = x_i + INTT(ExtProd(sel_i, y_i - x_i)) (the gadget
 * decomposition of y_i - x_i times the RGSW selector sel_i, in the NTT
 * domain, back to coefficient form), with no server handle and no
 * allocation.
 *   d_x, d_y      : n x 2N u64 device arrays, coefficient form mod q
 *   d_selectors   : n x 2 L_EP rows x 2N u64 device array, RGSW selector in
 *                   NTT form (the complete_selectors layout)
 *   d_out         : n x 2N u64 device array (may not alias the inputs)
 *   stream        : cudaStream_t to enqueue on (NULL = legacy default stream)
 * Working memory is one fixed array inside the library (about 3.9 MiB per
 * device that loads the library, held until process exit); n above
 * OPIR_NOALLOC_MAX_MUX is rejected with OPIR_ERR_INVALID_ARGUMENT. The first
 * call on each device sets up that device (looks up the array's device
 * address and copies the NTT tables into it with a synchronous cudaMemcpy),
 * so make the first call before any stream capture. Every call shares the
 * same array: calls whose work overlaps on the GPU (different streams, or
 * different host threads) race and must be serialised by the caller. Each
 * call overwrites every scratch word it reads, so nothing depends on what an
 * earlier call left behind. Only the CONFIG_N2048_K1_COMP parameter set. */
#define OPIR_NOALLOC_MAX_MUX 8
opir_status opir_ext_prod_mux_noalloc(const opir_params *params, uint32_t n,
                                      const uint64_t *d_x, const uint64_t *d_y,
                                      const uint64_t *d_selectors, uint64_t *d_out,
                                      void *stream);

/* ---- client-side batch operations ---------------------------------------
 * The two client steps of the protocol that scale with the number of queries
 * or responses, for one client (one ternary secret) at a time: query packing
 * (PirClient::fast_generate_query, src/client.cpp:107-225) and response
 * decryption (PirClient::decrypt_mod_q, src/client.cpp:364-410), plus the
 * client's session keys. The random samples stay with the caller. A client
 * handle holds the secret on one device; calls on one handle must not run
 * concurrently. */
typedef struct opir_client opir_client;

/* secret: N int8 coefficients in {-1, 0, 1} (the coefficient form of the
 * client's RlweSk, includes/rlwe.h:33-44). params: a database layout
 * (opir_params_init[_config]); the queries address that layout. */
opir_status opir_client_create(const opir_params *params, const int8_t *secret, int device,
                               opir_client **out);
void opir_client_destroy(opir_client *client);
const char *opir_client_last_error(const opir_client *client);

/* fast_generate_query for n plaintext indices (host array pt_idx, each below
 * num_pt, else OPIR_ERR_OUT_OF_RANGE) with the randomness given:
 *   d_a       : n x K N u64 device array, the uniform c1 of each query, limb
 *               k below q_k (the logical q when K = 1)
 *   d_e       : n x N int64 device array, the error of each query (shared by
 *               the limbs when K = 2)
 *   d_queries : n x 2 K N u64 device array, each [c0 (K N)][c1 (K N)] with
 *               c1 = a and c0 = -(a s + e) plus the packed plaintext (the
 *               one-hot's BFV lift and the selector gadget rows)
 * stream: cudaStream_t (NULL = legacy default stream). Equal, for equal
 * (secret, a, e), to the reference's query coefficient for coefficient. */
opir_status opir_client_generate_queries_device(opir_client *client, uint32_t n,
                                                const uint64_t *pt_idx, const uint64_t *d_a,
                                                const int64_t *d_e, uint64_t *d_queries,
                                                void *stream);

/* decrypt_mod_q for n responses:
 *   d_responses  : n x 2N u64 device array, coefficient form mod small_q as
 *                  PirClient::load_resp_from_stream yields (client.cpp:315-361)
 *   d_plaintexts : n x N u64 device array, each coefficient below t
 *   d_max_noise  : n u64 device array or NULL: the response's max noise
 *                  |phase - round(small_q m / t)| (client.cpp:389-407)
 * Under CONFIG_N2048_K1_COMP batches of 32 or more run on the tensor cores
 * (as do query batches of 32 or more in opir_client_generate_queries_device);
 * those calls synchronise `stream` before returning, to read the bounded
 * waits' error word of the tensor-core kernel. */
opir_status opir_client_decrypt_device(opir_client *client, uint32_t n,
                                       const uint64_t *d_responses, uint64_t *d_plaintexts,
                                       uint64_t *d_max_noise, void *stream);

/* create_session_keys (client.cpp:40-45) with the randomness given: the BV
 * key-switching keys for galois_k = N/2^i + 1, i < h (gen_bv_ks_key,
 * bv_keyswitch.cpp:191-276: row r = (B^r sigma_k(s) - a s + e, a) with
 * B = 2^base_log2_ks) and the RGSW encryption of s (generate_gsw_from_key,
 * client.cpp:25-38, gsw.cpp:359-422: row (half, r) = an encryption of zero
 * (-(a s + e), a) plus s B_key^(L_KEY-1-r) in polynomial `half`), every
 * polynomial then in the NTT domain -- the layouts opir_server_set_client_keys
 * takes.
 *   d_bv_a / d_bv_e   : h x L_KS x K N u64 (uniform, coefficient form) and
 *                       h x L_KS x N int64 (error) device arrays; NULL when h = 0
 *   d_gsw_a / d_gsw_e : 2 L_KEY x K N u64 and 2 L_KEY x N int64
 *   d_bv_keys         : h x L_KS x 2 x K N u64, each row [b][a]
 *   d_gsw_key         : 2 L_KEY x 2 x K N u64, each row [c0][c1]
 * Equal, for equal (secret, a, e), to the reference's keys. */
opir_status opir_client_keygen_device(opir_client *client, const uint64_t *d_bv_a,
                                      const int64_t *d_bv_e, const uint64_t *d_gsw_a,
                                      const int64_t *d_gsw_e, uint64_t *d_bv_keys,
                                      uint64_t *d_gsw_key, void *stream);

/* The same three calls on host arrays (same layouts and meaning, without the
 * d_ prefix), run on the handle's own stream; each returns once its results
 * are in host memory. max_noise may be NULL. */
opir_status opir_client_generate_queries(opir_client *client, uint32_t n, const uint64_t *pt_idx,
                                         const uint64_t *a, const int64_t *e,
                                         uint64_t *queries);
opir_status opir_client_decrypt(opir_client *client, uint32_t n, const uint64_t *responses,
                                uint64_t *plaintexts, uint64_t *max_noise);
opir_status opir_client_keygen(opir_client *client, const uint64_t *bv_a, const int64_t *bv_e,
                               const uint64_t *gsw_a, const int64_t *gsw_e, uint64_t *bv_keys,
                               uint64_t *gsw_key);

/* ---- tree PIR level selection ------------------------------------------
 * The full-binary-tree PIR layer of the reference (src/tree_index.cpp,
 * src/tree_query.cpp, src/tree_select.cpp): levels 0..L of a tree with
 * N = 2^L leaves, each level packed into R_l = 2^max(l - r, 0) plaintexts
 * (r = log2 n), one packed query expanded into an alpha one-hot of N0 = 2^a
 * ciphertexts plus b + r RGSW selectors. */

/* TreePirParams (includes/tree_index.h:23-55), g = 1. */
typedef struct {
  uint64_t N, L, n, g, rho, r, N0, a, P, B, b;
  uint64_t ell_beta, ell_gamma, w, h_q, W;
  uint64_t t;
} opir_tree_params;

typedef enum {
  OPIR_TREE_SINGLE = 0,          /* R_l = 1 */
  OPIR_TREE_COARSENED_ALPHA = 1, /* 1 < R_l < N0 */
  OPIR_TREE_ALPHA_BETA = 2       /* R_l >= N0 */
} opir_tree_case;

/* LevelPlan (includes/tree_index.h:76-92). */
typedef struct {
  uint64_t level, R;
  uint32_t select_case, reserved;
  uint64_t coarsen_count, beta_begin, beta_count, gamma_begin, gamma_count,
      projection_depth;
} opir_tree_level_plan;

/* make_tree_pir_params (src/tree_index.cpp:47-92) for any ring shape (pure
 * index math; moduli: n_moduli RNS moduli). Violations of
 * validate_tree_params (src/tree_index.cpp:93-150) ->
 * OPIR_ERR_INVALID_ARGUMENT. */
opir_status opir_tree_params_make(uint64_t L, uint64_t a, uint64_t n, uint64_t ell_beta,
                                  uint64_t ell_gamma, uint64_t t, const uint64_t *moduli,
                                  uint32_t n_moduli, opir_tree_params *out);
/* make_tree_pir_params_for_scheme (src/tree_query.cpp:42-62): n, t, the RNS
 * moduli and ell_beta = ell_gamma = L_EP from `scheme`, validated as
 * validate_tree_params (src/tree_index.cpp:93-150); a query expansion height
 * above the scheme's -> OPIR_ERR_INVALID_ARGUMENT. */
opir_status opir_tree_params_init(uint64_t L, uint64_t a, const opir_params *scheme,
                                  opir_tree_params *out);
/* build_level_plans (src/tree_index.cpp:177-225): L + 1 plans into `out`. */
opir_status opir_tree_level_plans(const opir_tree_params *tree, opir_tree_level_plan *out);
/* tree_query_expansion_params (src/tree_query.cpp:64-68): the query-shape
 * view {N0, b + r, h_q} a server needs for unpack_tree_query, which is
 * opir_server_expand_query + opir_server_complete_selectors on it. */
opir_status opir_tree_query_params(const opir_tree_params *tree, const opir_params *scheme,
                                   opir_params *out);
/* A device-resident tree level for select_level (src/tree_select.cpp:
 * 203-238): level `level` of `tree` with its R_l packed plaintexts
 * (pack_tree_level order, src/tree_select.cpp:55-75: R_l x n coefficients,
 * each < t). The handle is a server (opir_server_destroy releases it). */
opir_status opir_tree_level_create(const opir_params *scheme, const opir_tree_params *tree,
                                   uint64_t level, const uint64_t *plaintexts, int device,
                                   opir_server **out);
/* select_level (src/tree_select.cpp:203-238) for one expanded tree query:
 *   alpha          : N0 ciphertexts (the alpha one-hot A^(0), coefficient form)
 *   beta_selectors : b RGSW selectors (2 L_EP rows x ciphertext each, NTT
 *                    form, the complete_selectors layout); may be NULL when
 *                    the level's plan folds no beta bit
 *   out            : the selected ciphertext, coefficient form.
 * Bit for bit the reference's result: the coarsened pyramid and the
 * alpha-dimension products are one contraction over the N0 alpha
 * ciphertexts (the level's plaintexts replicated over the columns they
 * select), followed by the MSB-first beta fold of ext_prod_mux steps. */
opir_status opir_tree_select_level(opir_server *level, const uint64_t *alpha,
                                   const uint64_t *beta_selectors, uint64_t *out);

/* A whole device-resident tree (either parameter set): the query-shape server
 * that unpacks tree queries and one level database per level 0..L, all on
 * one device. A query is answered without host round trips between its
 * stages: expansion and selector completion on the query handle, then every
 * level's select_level on its own stream (levels overlap on the GPU), the
 * alpha ciphertexts and fold selectors passed device to device.
 *   level_plaintexts : L + 1 pointers, level l = R_l x n coefficients < t
 *                      (pack_tree_level order) */
typedef struct opir_tree opir_tree;
opir_status opir_tree_create(const opir_params *scheme, const opir_tree_params *tree,
                             const uint64_t *const *level_plaintexts, int device,
                             opir_tree **out);
void opir_tree_destroy(opir_tree *tree);
const char *opir_tree_last_error(const opir_tree *tree);
/* The client's BV keys (for the tree query's expansion height) and RGSW(s),
 * as opir_server_set_client_keys. */
opir_status opir_tree_set_client_keys(opir_tree *tree, uint64_t client_id,
                                      const uint64_t *bv_keys, const uint32_t *galois_ks,
                                      uint32_t n_keys, const uint64_t *gsw_key);
/* unpack_tree_query + select_level at every level for one packed tree query
 * (host buffers): selected = (L + 1) ciphertexts (2N u64 each, 4N under
 * CONFIG_N4096_K2_MP), level order, coefficient form -- bit for bit
 * opir_tree_select_level of each level. */
opir_status opir_tree_query(opir_tree *tree, uint64_t client_id, const uint64_t *query,
                            uint64_t *selected);

/* make_tree_query (src/tree_query.cpp:142-196) for n client coordinates on
 * the GPU, with a client handle (opir_client_create, any layout of the same
 * parameter set) and the randomness given: per query alpha (< N0), `groups`
 * selector bits (b beta bits, then r gamma bits, one byte each, n x groups),
 * the uniform c1 a (K N) and the error e (N); queries: n ciphertexts in the
 * opir_tree_query layout. Host arrays; returns when the queries are written. */
opir_status opir_client_generate_tree_queries(opir_client *client, const opir_tree_params *tree,
                                              uint32_t n, const uint64_t *alpha,
                                              const uint8_t *bits, uint32_t groups,
                                              const uint64_t *a, const int64_t *e,
                                              uint64_t *queries);

/* Library version string. */
const char *opir_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ONIONPIR_B200_H */
