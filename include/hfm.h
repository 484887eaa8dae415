/*
 * hfm.h — C ABI of haystackfm_b200, the B200 (sm_100a) engine for haystackfm's
 * batched query path: IUPAC backward search with sampled-SA locate, and the
 * bidirectional SMEM/MEM pipeline (find intervals, resolve SA positions, map to
 * reference boundaries).
 *
 * Plain C types only.  Every entry point returns an hfm status (0 = OK, < 0 =
 * error; message via hfm_last_error()).  Queries are encoded IUPAC codes 0..15
 * (src/alphabet.rs:3-52 of the reference), concatenated, with nq+1 u64 offsets.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * sriram98v/haystackfm).  Results are bit-exact with the reference CPU
 * count / locate / find_smems / find_mems on the same index bytes.
 */
#ifndef HFM_H
#define HFM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define HFM_OK 0
#define HFM_E_CUDA (-1)     /* CUDA runtime error (maps to FmIndexError::GpuError)          */
#define HFM_E_OOM (-2)      /* device or host allocation failed                             */
#define HFM_E_FORMAT (-3)   /* bad bincode / alphabet tag / inconsistent index (DeserializeError) */
#define HFM_E_ARG (-4)      /* invalid argument                                             */
#define HFM_E_TIMEOUT (-5)  /* the handle's deadline (hfm_set_timeout) passed while waiting    */
#define HFM_E_OVERFLOW (-6) /* a per-read work set outgrew the largest fallback capacity     */
#define HFM_E_WALK (-7)     /* an LF walk exceeded sample_rate steps (index inconsistent)   */
#define HFM_E_CHAR (-8)     /* a read holds a character outside the alphabet, or no read was
                               found (FmIndexError::InvalidCharacter)                        */

#define HFM_KIND_FM 0       /* FmIndex bytes        (src/fm_index/serialize.rs:13-52)       */
#define HFM_KIND_BIDIR 1    /* BidirFmIndex bytes   (src/fm_index/bidir_index.rs:183-210)   */

#define HFM_MODE_SMEM 0     /* src/gpu/mem_find.rs:9 */
#define HFM_MODE_MEM 1      /* src/gpu/mem_find.rs:10 */

typedef struct hfm_index hfm_index;   /* device-resident index, opaque */

#define HFM_FLAG_DEDUP_ALWAYS 1u  /* resolve repeated SA intervals once per call, always      */
#define HFM_FLAG_DEDUP_NEVER 2u   /* never deduplicate (default: when hits average >= 4 rows) */

typedef struct hfm_opts {
  int32_t device;          /* CUDA device ordinal (one index per GPU; replicate for multi-GPU) */
  uint32_t flags;          /* HFM_FLAG_* (0 = defaults)                                        */
} hfm_opts;

typedef struct hfm_index_info {
  uint32_t kind, text_len, num_sequences, sample_rate;
  uint32_t lookup_depth, alphabet_tag, num_lanes, encoding;
  uint64_t device_bytes;   /* HBM held by the device layout */
} hfm_index_info;

/* Locate result: per-query CSR of (seq_idx, pos_in_seq) pairs in the reference CPU
 * order (merged SA intervals ascending, rows ascending; src/fm_index/query.rs:22-39). */
typedef struct hfm_hits {
  uint32_t nq;
  uint32_t _pad;
  uint64_t total;          /* number of pairs                                   */
  uint64_t* offsets;       /* nq + 1                                            */
  uint32_t* counts;        /* exact FmIndex::count per query (uncapped)         */
  uint32_t* pairs;         /* 2 * total: seq_idx, pos_in_seq                    */
} hfm_hits;

/* One hit per SA interval of a MEM, as the reference GPU MemHit
 * (src/gpu/mem_hit.rs:6-19, src/fm_index/bidir_index.rs:452-468).  Hits of one MEM
 * are in ascending fwd_lo order; MEMs in ascending (query_start, query_end). */
typedef struct hfm_mem_hit {
  uint32_t query_start, query_end;
  uint32_t match_count;    /* SA interval size                                  */
  uint32_t truncated;      /* match_count > max_hits                            */
  uint32_t fwd_lo;         /* forward SA interval start                         */
  uint32_t n_pos;          /* positions resolved: min(match_count, max_hits), 0 without bounds */
  uint64_t pos_off;        /* first (ref_id, offset) pair in positions          */
} hfm_mem_hit;

typedef struct hfm_mem_out {
  uint32_t nq;
  uint32_t _pad;
  uint64_t n_hits, n_positions;
  uint64_t* hit_offsets;   /* nq + 1                                            */
  hfm_mem_hit* hits;       /* n_hits                                            */
  uint32_t* positions;     /* 2 * n_positions: ref_id, offset_within_ref        */
} hfm_mem_out;

/* Per-call device timings and work counters of the last query on a handle.  Times are
 * CUDA events recorded on the handle's stream around the phases and around the main
 * search kernel and the resolve kernel alone.  Work counters are filled only while
 * hfm_set_counters(idx, 1) is on (they slow the kernels). */
typedef struct hfm_stats {
  float ms_search, ms_resolve, ms_total;
  float ms_search_kernel, ms_resolve_kernel;
  uint32_t search_launches, resolve_launches, other_launches, fallback_reads;
  uint64_t occ_touches;      /* Occ record touches of the search kernels (incl. lookup reads) */
  uint64_t lf_calls;         /* LF-walk iterations of the resolve kernel (Occ + SA-marker touch each) */
  uint64_t rows_resolved;    /* positions resolved (one sa_vals read and one output pair each) */
  uint64_t hits_out;         /* MEM hit records written                                   */
  uint64_t rows_unique;      /* distinct rows walked after deduplication (0: no dedup)     */
} hfm_stats;

/* ---- index construction (replaces FmIndex::build_cpu_with + to_bytes,
 *      src/fm_index/mod.rs:95-195, src/fm_index/bidir_index.rs:53-80,
 *      src/fm_index/serialize.rs:13-26) ------------------------------------- */
typedef struct hfm_build_opts {
  uint32_t sa_sample_rate;   /* FmIndexConfig::sa_sample_rate (default 32)            */
  uint32_t lookup_depth;     /* FmIndexConfig::lookup_depth (reverse index always 0)  */
  uint32_t alphabet_tag;     /* 0 IupacDna, 1 ExactDna                                */
  uint32_t occ_encoding;     /* 0 Bitplane, 1 OneHot                                  */
  uint32_t threads;          /* host threads for construction (0 = all)               */
} hfm_build_opts;

/* codes: concatenated sequences (codes 1..15), seq_off[nseq+1]; headers: nseq C strings
 * or NULL ("seq_{i}" defaults).  Writes malloc'd bincode bytes (free with hfm_free). */
int hfm_build_index(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq,
                    const char* const* headers, const hfm_build_opts* opts, int kind,
                    uint8_t** bytes_out, size_t* len_out);

/* The same bytes as hfm_build_index, built on GPU `device` (replaces FmIndex::build /
 * BidirFmIndex::build, src/fm_index/mod.rs:209-284, src/fm_index/bidir_index.rs:91-116,
 * whose wgpu build is IUPAC-only with a 16-lane Occ table and no lookup table; this one
 * keeps build_cpu_with's contract).  Suffixes are sorted by prefix doubling over a device
 * radix sort; BWT, Occ records, sampled SA and lookup table are built on the device.
 * Needs about 39 bytes of device memory per text position while sorting. */
int hfm_build_index_gpu(const uint8_t* codes, const uint64_t* seq_off, uint32_t nseq,
                        const char* const* headers, const hfm_build_opts* opts, int kind, int device,
                        uint8_t** bytes_out, size_t* len_out);

/* ---- index load / free (replaces FmIndex::from_bytes / BidirFmIndex::from_bytes,
 *      src/fm_index/serialize.rs:32-52, src/fm_index/bidir_index.rs:195-210, and the
 *      per-call uploads of src/gpu/locate.rs:69-111, src/gpu/mem_find.rs:56-102,
 *      src/gpu/mem_resolve.rs:44-85) ---------------------------------------- */
int hfm_index_load(const uint8_t* bincode, size_t len, int kind, const hfm_opts* opts, hfm_index** out);
/* Device-layout blob (no counterpart in the reference): hfm_index_export_layout writes the
 * handle's device records — after the transform from the bincode records that
 * hfm_index_load makes on the host — to one malloc'd block (*bytes_out, released with
 * hfm_free); hfm_index_load_layout uploads such a block as it is, so a repeated load of a
 * genome-scale index is a read and a copy.  Every length is checked against the text
 * length and the blob size before any device work (HFM_E_FORMAT).  The blob is specific
 * to this library's version and is not the reference's bincode. */
int hfm_index_export_layout(hfm_index* idx, uint8_t** bytes_out, uint64_t* len_out);
int hfm_index_load_layout(const uint8_t* bytes, uint64_t len, const hfm_opts* opts, hfm_index** out);
void hfm_index_free(hfm_index* idx);
/* Device bytes a handle holds: its index layout (0 for a share) and its grow-only work
 * areas, pools and result arrays (reused across calls; freed with the handle).  For
 * budgeting HBM between handles; no counterpart in the reference. */
int hfm_index_device_bytes(const hfm_index* idx, uint64_t* index_bytes, uint64_t* work_bytes);
int hfm_index_info_get(const hfm_index* idx, hfm_index_info* out);
/* A second handle on the same device-resident index, with its own stream and work buffers
 * (no counterpart in the reference, whose process-wide context serialises every call,
 * src/gpu/context_cache.rs:5-19): calls on the two handles run concurrently without a
 * second copy of the index in HBM.  `idx` must outlive the shares; free each share with
 * hfm_index_free (it leaves the index's buffers to `idx`). */
int hfm_index_share(hfm_index* idx, hfm_index** out);

/* ---- queries, host buffers (the drop-in boundary) ------------------------ */

/* FmIndex::count over a batch (src/fm_index/query.rs:9-14). */
int hfm_count_batch(hfm_index* idx, const uint8_t* q, const uint64_t* q_off, uint32_t nq,
                    uint32_t* counts_out);

/* locate_batch_gpu (src/gpu/locate.rs:52-277) with the CPU semantics of
 * FmIndex::locate (src/fm_index/query.rs:22-39, lookup seeding and unbounded IUPAC
 * interval sets included).  max_hits > 0 keeps the first max_hits rows of every merged
 * interval (an extension: the reference locate has no cap); 0 = all rows. */
int hfm_locate_batch(hfm_index* idx, const uint8_t* q, const uint64_t* q_off, uint32_t nq,
                     uint32_t max_hits, hfm_hits** out);

/* BidirFmIndex::find_smems_gpu / find_mems_gpu (src/fm_index/bidir_index.rs:225-276,
 * 391-514) with the CPU find_smems / find_mems semantics (src/fm_index/smem.rs:71-124).
 * ref_bounds: exclusive end of each reference in the concatenated text (n_bounds = 0
 * skips position resolution, as the reference does). */
int hfm_mems_batch(hfm_index* idx, const uint8_t* q, const uint64_t* q_off, uint32_t nq,
                   uint32_t min_len, uint32_t mode, const uint32_t* ref_bounds, uint32_t n_bounds,
                   uint32_t max_hits, hfm_mem_out** out);

/* ---- queries, device buffers (reads already resident in HBM) -------------
 * Same semantics as above.  d_q / d_q_off are device pointers; results are written to
 * device memory owned by the handle and stay valid until the next call on it.
 * Ordering: every call runs on the handle's own stream (created non-blocking, so it does
 * not wait for the legacy default stream or for any stream of the caller).  Device inputs
 * and caller-owned device outputs must be complete before the call is made (synchronize
 * the stream that wrote them); the call returns after its device work has finished, so
 * its outputs are ready for any stream when it returns. */
typedef struct hfm_dev_hits {
  uint32_t nq; uint32_t _pad; uint64_t total;
  uint64_t* d_offsets; uint32_t* d_counts; uint32_t* d_pairs;
} hfm_dev_hits;
typedef struct hfm_dev_mems {
  uint32_t nq; uint32_t _pad; uint64_t n_hits, n_positions;
  uint64_t* d_hit_offsets; hfm_mem_hit* d_hits; uint32_t* d_positions;
} hfm_dev_mems;

int hfm_count_batch_device(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq,
                           uint32_t* d_counts_out);
int hfm_locate_batch_device(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq,
                            uint32_t max_hits, hfm_dev_hits* out);
int hfm_mems_batch_device(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq,
                          uint32_t min_len, uint32_t mode, const uint32_t* ref_bounds, uint32_t n_bounds,
                          uint32_t max_hits, hfm_dev_mems* out);

/* Allocation-free count (no counterpart in the reference).  Same results as
 * hfm_count_batch_device, for callers that must not let a library allocate GPU memory:
 * frameworks that own the device's memory through their own pool, and latency-bound
 * serving loops that cannot absorb cudaMalloc's synchronisation.  Its work area is one
 * static 17 MiB device array inside libhfm.so (present on every GPU that loads the library
 * until exit) instead of handle buffers; inputs and output are the caller's device memory.
 * Limits: nq <= 1,048,576 per call (else HFM_E_ARG); interval sets of at most 2,048
 * intervals per query (else HFM_E_OVERFLOW, use hfm_count_batch).  All calls share the
 * array: calls that overlap on the GPU race, so serialise them.  The first call on a
 * device looks up the array's device address; make it before any stream capture. */
int hfm_count_batch_noalloc(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq,
                            uint32_t* d_counts_out);

/* Scheduled SMEM/MEM search (no counterpart in the reference): the hook of the learned
 * read scheduler.  Results are identical to hfm_mems_batch_device for every schedule.
 *   d_order    device permutation of 0..nq-1: the order in which the persistent per-thread
 *              kernel takes reads from its queue (NULL: 0..nq-1).  Checked on the device;
 *              anything else is HFM_E_ARG before any search runs.
 *   n_warp     the first n_warp reads of d_order skip the per-thread kernel and go to the
 *              warp-per-read kernel (reads predicted to outgrow per-thread interval sets).
 *   d_work_log device array of 4*nq u32, or NULL.  When set, the call runs the counting
 *              kernel variants and logs the exact work of each read i:
 *              [4i] Occ record touches (backward and forward extension steps, every pass),
 *              [4i+1] MemHits reported, [4i+2] positions reported,
 *              [4i+3] bit 0: the read left the fast per-thread pass (its candidate list
 *              or an interval set outgrew the fast path, or n_warp routed it); bit 1: it
 *              ran on the warp-per-read kernel. */
typedef struct hfm_sched {
  const uint32_t* d_order;
  uint32_t n_warp;
  uint32_t _pad;
  uint32_t* d_work_log;
} hfm_sched;
int hfm_mems_batch_device_sched(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq,
                                uint32_t min_len, uint32_t mode, const uint32_t* ref_bounds, uint32_t n_bounds,
                                uint32_t max_hits, const hfm_sched* sched, hfm_dev_mems* out);

/* CUDA-graph-captured SMEM/MEM pass chain (no counterpart in the reference, whose batch
 * search reads counts back to the host between its passes, src/gpu/mem_find.rs:213-244).
 * hfm_mems_graph_create captures, for batches of nq reads at the fixed device addresses
 * d_q / d_q_off, the whole search-CSR-resolve chain of hfm_mems_batch_device into one CUDA
 * graph: every pass runs over capacities fixed at capture (the handle's pool capacities,
 * as hfm_mems_reserve set them; max_positions resolved positions; long-read segments for
 * up to max_bases codes per batch) and reads its counts from device memory, so nothing
 * waits on the host inside the chain.  The graph works on a private copy of the handle's
 * buffers and stream and shares the index.  hfm_mems_graph_launch replays it for the reads
 * the caller has written to d_q / d_q_off (nq reads, offsets from 0): it reads the batch's
 * length first, replays, and checks the overflow flags; a batch that outgrew a capacity is
 * rerun on the adaptive chain (same results) and the graph is captured again with the
 * grown capacities (*replayed = 0; 1 when the replay's outputs were returned).  Outputs
 * are those of hfm_mems_batch_device, in the graph's own buffers, valid until the next
 * launch.  Calls on one graph must not overlap. */
typedef struct hfm_graph hfm_graph;
int hfm_mems_graph_create(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq, uint64_t max_bases,
                          uint32_t min_len, uint32_t mode, const uint32_t* ref_bounds, uint32_t n_bounds,
                          uint32_t max_hits, uint64_t max_positions, hfm_graph** out);
int hfm_mems_graph_launch(hfm_graph* g, hfm_dev_mems* out, uint32_t* replayed);
void hfm_mems_graph_free(hfm_graph* g);
/* Replays and fallbacks so far, and the reasons of the last launch's fallback (0: it was
 * replayed): HFM_GRAPH_* bits.  A warp-tier set overflow also quadruples that tier's set
 * capacity for the next capture. */
#define HFM_GRAPH_BASES 1u        /* the batch has more codes than the segment capacity   */
#define HFM_GRAPH_INTERVALS 2u    /* candidate-interval pool                              */
#define HFM_GRAPH_HITS 4u         /* MemHit pool                                          */
#define HFM_GRAPH_SEGMENTS 8u     /* long-read segment candidate pool                     */
#define HFM_GRAPH_WARP_SETS 16u   /* a read's interval set outgrew the warp tier          */
#define HFM_GRAPH_POSITIONS 32u   /* positions (or distinct positions) past the capacity  */
#define HFM_GRAPH_LOCATE 64u      /* the locate chain outgrew one of its capacities       */
int hfm_mems_graph_info(const hfm_graph* g, uint32_t* replays, uint32_t* fallbacks, uint32_t* last_reason);
/* Adds the locate chain of hfm_locate_batch_device (backward search, merged intervals,
 * resolve) for nq queries at fixed device addresses to the graph, ahead of its SMEM chain,
 * so that one replay runs both (the whole batched query step of the reference's
 * `query` and `mem`/`smem` paths, fm_index.rs and bidir.rs, without a host round trip
 * between them).  max_intervals / max_positions: capacities of the merged-interval pool and
 * of the resolved positions; a batch past either (or past the warp tier's set) is rerun on
 * the adaptive chain with the same results and the capacities grow.  The locate result of
 * the last hfm_mems_graph_launch is read with hfm_mems_graph_locate_result; it is that of
 * hfm_locate_batch_device for the same queries, in the graph's own buffers, valid until
 * the next launch. */
int hfm_mems_graph_add_locate(hfm_graph* g, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq,
                              uint32_t max_hits, uint64_t max_intervals, uint64_t max_positions);
int hfm_mems_graph_locate_result(const hfm_graph* g, hfm_dev_hits* out);

/* Pre-sizes a handle's SMEM/MEM work pools and result arrays for a batch of nq reads
 * expected to produce `intervals` candidate intervals, `hits` MemHits and `positions`
 * resolved positions (no counterpart in the reference, which counts every batch on the
 * device, downloads the counts and allocates before a second pass; src/gpu/mem_find.rs:
 * 213-244, src/fm_index/bidir_index.rs:442-514).  The learned read-cost model calls it
 * with its predicted totals, so the search runs once with no count pass and no buffer
 * growth; a batch that outgrows the reservation is rerun with grown pools (same results).
 * Buffers only grow. */
int hfm_mems_reserve(hfm_index* idx, uint32_t nq, uint64_t intervals, uint64_t hits, uint64_t positions);

/* ---- learned read-cost model (no counterpart in the reference) -------------
 * A 258 -> 128 -> 128 -> 3 ReLU MLP (BF16 weights and activations, FP32 accumulation)
 * predicting, per read, log1p of the exact SMEM kernel's work log (hfm_sched.d_work_log):
 * Occ touches, MemHits, positions.  Input row (HFM_MLP_IN_PAD BF16 values): 256 4-mer
 * frequencies x[f] = 256*c_f/V - 1 (V = 4-mers without an ambiguity code; all 0 when
 * V == 0), x[256] = (log2(len+1) - 10)/4, x[257] = (len-3-V)/(len-3) (0 when len < 4),
 * zeros to the end.  Parameters (FP32, in this order): W1[128][272], b1[128],
 * W2[128][128], b2[128], W3[3][128], b3[3]; W1 columns 258..271 multiply zero inputs.  Training runs the model's own forward and backward CUDA
 * kernels and Adam (lr as given, betas 0.9 / 0.999, eps 1e-8) on the MSE of the outputs.
 * Every call completes its work before returning; device arrays must be 16-byte aligned. */
#define HFM_MLP_IN_PAD 272
#define HFM_MLP_HIDDEN 128
#define HFM_MLP_OUT 3
#define HFM_MLP_NPARAM (128 * 272 + 128 + 128 * 128 + 128 + 3 * 128 + 3)
typedef struct hfm_mlp hfm_mlp;
int hfm_mlp_create(int device, uint64_t seed, hfm_mlp** out);      /* He-uniform init from seed */
void hfm_mlp_free(hfm_mlp* m);
int hfm_mlp_set_params(hfm_mlp* m, const float* params);          /* host, HFM_MLP_NPARAM; resets Adam */
int hfm_mlp_get_params(hfm_mlp* m, float* params);                /* host, HFM_MLP_NPARAM */
void* hfm_mlp_stream(hfm_mlp* m);
/* d_x[nq][HFM_MLP_IN_PAD] (BF16 bits) from encoded reads */
int hfm_mlp_features(hfm_mlp* m, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq, uint16_t* d_x);
/* d_y[n][3] = model(d_x) */
int hfm_mlp_forward(hfm_mlp* m, const uint16_t* d_x, uint32_t n, float* d_y);
/* features + forward: d_y[nq][3] predicted log1p(touches, MemHits, positions) */
int hfm_mlp_predict(hfm_mlp* m, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq, float* d_y);
/* gradient of the MSE over all n rows (one batch) into d_grad[HFM_MLP_NPARAM]; *loss = MSE */
int hfm_mlp_grad(hfm_mlp* m, const uint16_t* d_x, const float* d_t, uint32_t n, float* d_grad, float* loss);
/* Adam over shuffled mini-batches (Fisher-Yates order from seed); loss_per_epoch[epochs] or NULL */
int hfm_mlp_train(hfm_mlp* m, const uint16_t* d_x, const float* d_t, uint32_t n, uint32_t epochs,
                  uint32_t batch, float lr, uint64_t seed, float* loss_per_epoch);
/* Schedule for hfm_mems_batch_device_sched: d_order = reads binned by predicted Occ
 * touches (4096 bins, costliest first); reads predicted to report at least warp_min_hits
 * MemHits (<= 0: none) come first and are counted in *n_warp (routed to the warp kernel).
 * Within a bin the order is unspecified; results never depend on it. */
int hfm_mlp_schedule(hfm_mlp* m, const float* d_y, uint32_t nq, float warp_min_hits, uint32_t* d_order,
                     uint32_t* n_warp);

/* Random-access ceiling of GPU `device` (no counterpart in the reference): independent
 * loads of `span` (32, 64 or 96: a narrow Occ record, a half, a wide record) bytes at
 * uniformly random span-aligned offsets of a buffer_bytes device buffer (>= 64 MiB; it is
 * allocated and freed by the call), 256-288 bytes in flight per thread on 8 x 256 threads
 * per SM.  *gbs_out = bytes loaded / second
 * (CUDA events), *ms_out (may be NULL) = one launch. */
int hfm_probe_gather(int device, uint64_t buffer_bytes, uint32_t span, float* gbs_out, float* ms_out);

/* ---- read ingest (host) ---------------------------------------------------- */
/* Text of reads -> the packed batch every query entry point takes (codes 1..15 of
 * src/alphabet.rs:54-94, either case, U as T; offsets[n + 1] with offsets[0] = 0).
 * format: HFM_READS_FASTA follows the reference's sequence reader (src/wasm/js_api.rs:18-68):
 * `>` lines start a record whose non-blank lines are concatenated, blank lines are skipped,
 * and lines before any header are one read each (no read at all: HFM_E_CHAR).
 * HFM_READS_FASTQ: four-line records (`@name`, sequence, `+...`, quality), blank lines
 * between records skipped, a malformed record is HFM_E_FORMAT with its line number.
 * HFM_READS_AUTO: FASTQ when the first non-blank character is `@`, else FASTA.  Lines
 * end at \n, \r\n or \r; white space around a line is ignored.  A character outside
 * the alphabet (`$` included) is HFM_E_CHAR, naming the character, its read and position.
 * threads: host threads for the encoding (0 = all).  *out is one block released with
 * hfm_free.  No counterpart in the reference's GPU path (which takes encoded
 * DnaSequence values); it replaces the caller-side parse + encode loop. */
#define HFM_READS_AUTO 0u
#define HFM_READS_FASTA 1u
#define HFM_READS_FASTQ 2u
typedef struct hfm_reads {
  uint64_t n;          /* reads                       */
  uint64_t n_codes;    /* total codes (offsets[n])    */
  uint64_t* offsets;   /* n + 1 entries               */
  uint8_t* codes;
} hfm_reads;
int hfm_parse_reads(const char* text, uint64_t len, uint32_t format, uint32_t threads, hfm_reads** out);

/* ---- misc ----------------------------------------------------------------- */
void hfm_free(void* p);                    /* frees hfm_hits*, hfm_mem_out*, hfm_reads*, build bytes */
const char* hfm_last_error(void);          /* thread-local message of the last failure   */
void* hfm_index_stream(hfm_index* idx);    /* the handle's cudaStream_t (for event timing) */
int hfm_last_stats(const hfm_index* idx, hfm_stats* out);
int hfm_set_counters(hfm_index* idx, int enable);  /* per-read work counters on/off (default off) */

/* Host-side deadline for the waits inside every call on the handle (no counterpart in the
 * reference, whose wgpu calls block without a limit; it stands in for the device watchdog
 * of FmIndexError::GpuError).  ms = 0 (default): wait without a limit.  When a wait passes
 * the deadline the call returns HFM_E_TIMEOUT at once: its outputs are undefined and a
 * device-to-host copy it issued may still land in its output later (hfm_count_batch's
 * counts_out included) until the next call on the handle, which first drains the abandoned
 * work; the handle stays usable. */
int hfm_set_timeout(hfm_index* idx, uint32_t ms);

/* Tunable parameters of the SMEM/MEM search and their autotuner (no counterpart in the
 * reference, whose shaders run a fixed workgroup_size(64), shaders/mem_find.wgsl:364-372).
 * Results never depend on them.
 *   mems_variant      persistent fast pass with 32-entry candidate lists in local memory (2)
 *                     or 1024-entry lists in global memory (3, default), 8 resident blocks
 *                     per SM; 4: the plain launch — one thread per read over a grid the size
 *                     of the batch, sets and candidates in local memory, a count pass whose
 *                     totals are read back to size the outputs before the write pass (the
 *                     reference GPU search's structure, src/gpu/mem_find.rs:213-244), kept
 *                     as the baseline.
 *   seg_len           SMEM reads longer than 2*seg_len are swept in seg_len-position segments
 *                     (multiple of 32 in 64..4096, default 512).
 *   queue_chunk       reads a per-thread kernel takes from its device work queue per atomic
 *                     (1..64, default 1).
 *   read_order        0 (default): the SMEM queue in the caller's read order (or the order of
 *                     hfm_mems_batch_device_sched); 1: reads queued in the order of their first
 *                     16 codes (a device radix sort; per-thread kernels only), so that reads
 *                     sharing a prefix — and the reference windows it selects — share a warp.
 *   threads_per_read  1 (default): a thread per read; 4, 8 or 16: every read on a group of
 *                     that many lanes (sub-warp kernel, the fast pass's set capacities; a
 *                     read that outgrows them goes on to the warp tier); 32: every read on
 *                     the warp-per-read kernel (the lanes of a group share each interval set).
 * hfm_autotune_mems times the search of a sample batch under each of the HFM_TUNE_CANDIDATES
 * settings {variant, seg_len, chunk, threads, order}: {3,512,1,1,0}, {3,256,1,1,0},
 * {3,1024,1,1,0}, {2,512,1,1,0}, {3,512,4,1,0}, {3,512,16,1,0}, {3,512,1,4,0}, {3,512,1,8,0},
 * {3,512,1,32,0}, {3,512,1,1,1}, {3,1024,1,1,1} — best of `reps` runs after a warm-up run,
 * by CUDA events on the handle's stream; it keeps the fastest on the handle, writes it to
 * *best, and the candidates' times to times_ms[HFM_TUNE_CANDIDATES] when non-NULL. */
#define HFM_TUNE_CANDIDATES 11
typedef struct hfm_tuning {
  uint32_t mems_variant;
  uint32_t seg_len;
  uint32_t queue_chunk;
  uint32_t threads_per_read;
  uint32_t read_order;
} hfm_tuning;
int hfm_get_tuning(const hfm_index* idx, hfm_tuning* out);
int hfm_set_tuning(hfm_index* idx, const hfm_tuning* t);
int hfm_autotune_mems(hfm_index* idx, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq, uint32_t min_len,
                      uint32_t mode, const uint32_t* ref_bounds, uint32_t n_bounds, uint32_t max_hits,
                      uint32_t reps, hfm_tuning* best, float* times_ms);

#ifdef __cplusplus
}
#endif
#endif /* HFM_H */
