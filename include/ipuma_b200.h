/*
 * ipuma_b200.h -- C ABI of the B200 batched Smith-Waterman (Gotoh) engine.
 *
 * Plain C: POD structs, raw pointers and sizes; no exceptions cross it.
 * Every entry point returns IPUMA_OK (0) or a negative IPUMA_ERR_* code;
 * ipuma_last_error() returns the message of the last failure on the calling
 * thread.  The C++ drop-in layer (ipuma-lib_b200/host, namespace ipu) is
 * built on these calls and rethrows failures as std::runtime_error with the
 * reference's messages.
 *
 * Reference interfaces replaced (paths relative to the ipuma-lib tree):
 *   ipuma_sw_config         ipu::SWConfig              src/ipu_config.h:11-19
 *   ipuma_algo_config       ipu::IPUAlgoConfig         src/ipu_config.h:21-42
 *   ipuma_gpu_create        SWAlgorithm::SWAlgorithm   src/ipu_batch_affine.cpp:372-403
 *                           (device attach ipu_base.cpp:127-148, engine build
 *                           ipu_batch_affine.cpp:388-400, executor :992-1012)
 *   ipuma_gpu_destroy       SWAlgorithm::~SWAlgorithm  src/ipu_batch_affine.cpp:1014-1022
 *   ipuma_gpu_run_buffer    prepared_remote_compare    src/ipu_batch_affine.cpp:558-562
 *                           (one engine run over the Seqs||Meta wire buffer,
 *                           FillCallback/RecvCallback :32-144, program :340-355)
 *   ipuma_gpu_submit_buffer async_submit_prepared_remote_compare  :496-506
 *   ipuma_gpu_join          blocking_join_prepared_remote_compare :508-556
 *   ipuma_gpu_poll          (non-blocking form of Job::join, :489-494)
 *   ipuma_gpu_compare       compare_local minus the host partitioning
 *                           (:564-663): pairs straight from a code array
 *   ipuma_gpu_compare_packed  the same with 2-, 4- or 5-bit packed codes
 *   ipuma_gpu_compare_device  the same with device-resident buffers
 *   ipuma_gpu_compare_device_packed  device-resident packed codes
 *   ipuma_pack_codes        (no counterpart: the reference stores one byte
 *                           per residue, fill_input_buffer :874-877)
 *   ipuma_encode            swatlib::Encoding::encode  src/swatlib/encoding.cpp:38-60
 *   ipuma_select_matrix     swatlib::selectMatrix      src/swatlib/similarity.cpp:89-105
 */
#ifndef IPUMA_B200_H
#define IPUMA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define IPUMA_OK 0
#define IPUMA_ERR_INVALID_ARG -1   /* bad pointer, size or config value     */
#define IPUMA_ERR_CUDA -2          /* a CUDA runtime call failed            */
#define IPUMA_ERR_NO_DEVICE -3     /* no usable CUDA device                 */
#define IPUMA_ERR_TOO_LONG -4      /* a sequence exceeds a stated maximum   */
#define IPUMA_ERR_OUT_OF_BUCKETS -5 /* partitioning capacity exhausted      */
#define IPUMA_ERR_BAD_SEQUENCE -6  /* a character has no code in the alphabet */
#define IPUMA_ERR_TIMEOUT -7       /* a bounded wait expired                */
#define IPUMA_ERR_NO_MEMORY -8     /* admission refused: not enough memory  */
#define IPUMA_ERR_UNKNOWN_JOB -9   /* job id not issued by this engine      */
#define IPUMA_ERR_DEVICE -10       /* a kernel reported an error status     */
#define IPUMA_ERR_CLOSED -11       /* engine or queue already closed        */

/* ---- enums, numbered like the reference's ------------------------------ */
/* swatlib::Similarity (src/swatlib/similarity.h:108-113) */
#define IPUMA_SIM_NUCLEIC_ACID 0
#define IPUMA_SIM_BLOSUM50 1
#define IPUMA_SIM_BLOSUM62 2
#define IPUMA_SIM_SIMPLE 3
/* swatlib::DataType (src/swatlib/encoding.h:12-16) */
#define IPUMA_DT_NUCLEIC_ACID 0
#define IPUMA_DT_AMINO_ACID 1
#define IPUMA_DT_STRING 2
/* ipu::VertexType (src/types.h:19) -- accepted, all compute the same result */
#define IPUMA_VTYPE_CPP 0
#define IPUMA_VTYPE_ASSEMBLY 1
#define IPUMA_VTYPE_MULTI 2
#define IPUMA_VTYPE_MULTIASM 3
/* ipu::Algorithm (src/types.h:21) -- host bucket policy of prepare_remote */
#define IPUMA_FILL_FIRST 0
#define IPUMA_FILL_ROUND_ROBIN 1
#define IPUMA_FILL_GREEDY 2

/* ---- configuration ------------------------------------------------------ */
/* ipu::SWConfig (src/ipu_config.h:11-19); defaults 0, -1, 1, -1, -1, NA, NA. */
typedef struct ipuma_sw_config {
  int32_t gap_init;
  int32_t gap_extend;
  int32_t match_value;
  int32_t mismatch_value;
  int32_t ambiguity_value;
  int32_t similarity; /* IPUMA_SIM_* */
  int32_t datatype;   /* IPUMA_DT_*  */
} ipuma_sw_config;

/* ipu::IPUAlgoConfig (src/ipu_config.h:21-42); defaults 1, 300, 20, 3000,
 * cpp, fillFirst, false, false, 1, 0.  tiles_used * max_batches comparison
 * slots and bufsize bytes of sequence per tile define the wire buffer of
 * ipuma_gpu_run_buffer; the other API ignores the layout fields. */
typedef struct ipuma_algo_config {
  int32_t tiles_used;
  int32_t max_ab;
  int32_t max_batches;
  int32_t bufsize;
  int32_t vtype;
  int32_t fill_algo;
  int32_t forward_only;
  int32_t use_remote_buffer;
  int32_t transmission_programs;
  int32_t io_tiles;
} ipuma_algo_config;

/* One comparison of the pair API: A = codes[a_off .. a_off + a_len), B likewise.
 * Codes are the swatlib codes of the engine's datatype (ipuma_encode). */
typedef struct ipuma_pair {
  int64_t a_off;
  int64_t b_off;
  int32_t a_len;
  int32_t b_len;
} ipuma_pair;

/* Timing and work counters of the last completed call on an engine. */
#define IPUMA_MAX_TIMED 24  /* launches ipuma_stats can time per call */

typedef struct ipuma_stats {
  double kernel_ms;     /* device time of the alignment kernels (CUDA events) */
  double total_ms;      /* device time including copies                      */
  int64_t cells;        /* sum of |A|*|B| (forward pass, ipuma's definition) */
  int64_t pairs;
  int64_t s32_pairs;    /* pairs the binning sent to the s32 or hybrid class
                           (main-diagonal score above the 16-bit limit)      */
  int64_t overflow_reruns; /* s16x2 pairs that were rerun in 32-bit          */
  int32_t launches;     /* kernels launched by the call                      */
  int32_t used_graph;   /* 1 when the call replayed a captured CUDA graph     */
  /* With option "time_launches" = 1: device time and forward-pass cells of
   * each alignment-kernel launch of the call, in launch order. */
  int32_t n_timed;
  int32_t timed_kind[IPUMA_MAX_TIMED];   /* IPUMA_KERNEL_* */
  double timed_ms[IPUMA_MAX_TIMED];
  int64_t timed_cells[IPUMA_MAX_TIMED];
  /* ipuma_gpu_compare: chunks the batch was split into for upload/compute
   * overlap (1 = one upload, then the kernels). */
  int32_t chunks;
  /* With option "trace" = 1: for each class launch of the batched pipeline
   * that ran (concurrently, as in production), the device time of its
   * first block's start and of its last warp's end, in ms from the call's
   * first start, and its forward-pass cells. */
  int32_t n_trace;
  int32_t trace_kind[IPUMA_MAX_TIMED];   /* IPUMA_KERNEL_* */
  double trace_start_ms[IPUMA_MAX_TIMED];
  double trace_end_ms[IPUMA_MAX_TIMED];
  int64_t trace_cells[IPUMA_MAX_TIMED];
  /* Host-buffer calls (ipuma_gpu_compare, ipuma_gpu_compare_packed): host
   * wall time of the descriptor check (bounds, maxima, code ranges per
   * chunk) and of the whole call. */
  double host_check_ms;
  double host_wall_ms;
} ipuma_stats;

/* Kernel kinds reported in ipuma_stats.timed_kind.  S16_L<lanes>_K<k>:
 * s16x2 lanes (two pairs per lane group), <lanes> lanes per group, <k> A
 * columns per lane. */
#define IPUMA_KERNEL_S32_K16 0     /* s32 lanes, 32 lanes, 16 columns       */
#define IPUMA_KERNEL_S16_L16_K4 1
#define IPUMA_KERNEL_S16_L16_K8 2
#define IPUMA_KERNEL_S16_L16_K12 3
#define IPUMA_KERNEL_S16_L16_K16 4
#define IPUMA_KERNEL_S16_L32_K12 5
#define IPUMA_KERNEL_S16_L32_K16 6
#define IPUMA_KERNEL_S32_RERUN 7   /* s32 rerun of 16-bit give-ups          */
#define IPUMA_KERNEL_PLAIN 8       /* one-launch-per-batch wire kernel      */
#define IPUMA_KERNEL_EXACT 9       /* per-thread exact kernel               */
#define IPUMA_KERNEL_S16_T_K16 10  /* signed s16x2, one thread per two pairs, 16-column strips */
#define IPUMA_KERNEL_S16_L16_K6 11
#define IPUMA_KERNEL_S16_L16_K10 12
#define IPUMA_KERNEL_S16_L16_K14 13
#define IPUMA_KERNEL_S16_L16_K5 14
#define IPUMA_KERNEL_S16_L16_K7 15
#define IPUMA_KERNEL_S16_L16_K9 16
#define IPUMA_KERNEL_S16_L16_K11 17
#define IPUMA_KERNEL_S16_L16_K13 18
#define IPUMA_KERNEL_S16_L16_K15 19
#define IPUMA_KERNEL_S16_HYBRID 20 /* scores above int16: strips in biased 16-bit halves (score - 31744,
                                      scores up to 65535 - 1024 - max(sim)) while safe, then s32 */
#define IPUMA_KERNEL_PLAIN_S16 21  /* one-launch-per-batch wire kernel, 16-bit lanes */
/* 8-lane groups (four per warp), used instead of S16_L16_K4 .. _K8 of the
 * same strip widths when the codes are 2-bit (four-row profiles) */
#define IPUMA_KERNEL_S16_L8_K8 22
#define IPUMA_KERNEL_S16_L8_K10 23
#define IPUMA_KERNEL_S16_L8_K12 24
#define IPUMA_KERNEL_S16_L8_K14 25
#define IPUMA_KERNEL_S16_L8_K16 26
#define IPUMA_KERNEL_S16_TEAM 27   /* s16x2, 512-column strips shared by a team of warps (one block per
                                      two pairs; long pairs of small batches) */

typedef struct ipuma_engine ipuma_engine;

/* ---- library ------------------------------------------------------------ */
const char* ipuma_last_error(void);
const char* ipuma_version(void);
/* Number of CUDA devices (0 when none is usable). */
int32_t ipuma_device_count(void);
/* Page-locked host memory for wire buffers (uploads at full bus speed, and
 * results are copied straight into it); *out = NULL when bytes = 0. */
int ipuma_host_alloc(size_t bytes, void** out);
void ipuma_host_free(void* p);

/* Host-only helpers (no GPU needed). */
/* Packs n codes for the packed compare calls into out[ceil(n * bits / 8)],
 * a little-endian bit stream: residue r in bits [bits*r, bits*r + bits).
 * bits = 5 takes codes < 32 (every amino-acid code, 0..24), bits = 4 codes
 * < 16 (nucleic acids with IUPAC codes), bits = 2 A, T, C, G (codes 1..4,
 * stored as code - 1); any other code gives IPUMA_ERR_BAD_SEQUENCE. */
int ipuma_pack_codes(const uint8_t* codes, size_t n, int32_t bits, uint8_t* out);
/* Encodes n chars into codes; unknown NA characters (code 16, which has no
 * row in the 16x16 NA matrix) are rejected with IPUMA_ERR_BAD_SEQUENCE. */
int ipuma_encode(int32_t datatype, const char* s, size_t n, uint8_t* out);
/* Writes the m x n substitution matrix (row = A code, column = B code). */
int ipuma_select_matrix(int32_t similarity, int32_t match, int32_t mismatch, int32_t ambiguity,
                        int8_t* out, size_t out_cap, int32_t* m, int32_t* n);
/* Size of the wire input buffer in int32 words
 * (IPUAlgoConfig::getInputBufferSize32b, src/ipu_config.cpp:6-14). */
int64_t ipuma_input_buffer_words(const ipuma_algo_config* algo);

/* ---- engine ------------------------------------------------------------- */
int ipuma_gpu_create(const ipuma_sw_config* sw, const ipuma_algo_config* algo, int32_t device,
                     ipuma_engine** out);
void ipuma_gpu_destroy(ipuma_engine* e);

/* Engine options:
 *   "scheduler"   0 = persistent cost-binned engine (default), 1 = plain
 *                 one-launch-per-batch kernel (wire-buffer API only)
 *   "plain_lanes" lanes of the plain kernel: 32 = one comparison slot per
 *                 warp in s32 lanes (default), 16 = two consecutive slots
 *                 per warp in s16x2 halves, a slot that could leave int16
 *                 redone in s32 by the same warp (IPUMA_KERNEL_PLAIN_S16)
 *   "graphs"      1 = capture and replay CUDA graphs for repeated shapes
 *   "tile_k"      0 = kernel class by |A| (default); 1..6 = every pair
 *                 through s16x2 class IPUMA_KERNEL_S16_* (value = kind),
 *                 7 = every pair through IPUMA_KERNEL_S16_T_K16, 8, 9, 10 =
 *                 IPUMA_KERNEL_S16_L16_K6, _K10, _K14, 11 .. 16 =
 *                 IPUMA_KERNEL_S16_L16_K5, _K7, _K9, _K11, _K13, _K15,
 *                 17 .. 21 = IPUMA_KERNEL_S16_L8_K8, _K10, _K12, _K14, _K16,
 *                 24 = every pair through strip teams (IPUMA_KERNEL_S16_TEAM)
 *   "concurrent"  3 = by batch size (default): mode 1 below 48,000 pairs,
 *                 mode 2 above; 2 = class launches alternate between two
 *                 streams, so each starts on the SMs the previous one
 *                 frees; 1 = all classes at once, each on a share of the
 *                 SMs proportional to its modelled work; 0 = one launch
 *                 after the other (always the case with time_launches)
 *   "latency_share" share of the batch's modelled time (per mille,
 *                 default 60) one pair's item may take in its class; a
 *                 pair over it takes a class that finishes it sooner
 *   "hybrid"      1 = pairs whose score can pass int16 run their strips
 *                 in biased 16-bit halves while a strip's values provably
 *                 fit, then in s32 (IPUMA_KERNEL_S16_HYBRID, default);
 *                 0 = all in s32
 *   "thread_class" 1 = the per-thread class IPUMA_KERNEL_S16_T_K16 may be
 *                 chosen for pairs that are small relative to the batch,
 *                 0 = never (default) unless tile_k forces it
 *   "time_launches" 1 = time every alignment-kernel launch (ipuma_stats)
 *   "trace"       1 = record when each class launch of the pipeline starts
 *                 and ends on the device, launches running concurrently
 *                 as usual (ipuma_stats trace_*)
 *   "autotune"    1 = measure the kernel-class rates before the first batch
 *                 (default), 0 = built-in rates unless ipuma_gpu_autotune
 *   "long_a"      |A| above which a pair takes the widest s16x2 class
 *                 (default 3072): long pairs are latency-bound
 *   "team_warps"  warps of a strip team (IPUMA_KERNEL_S16_TEAM): 2..8
 *                 (default 8; fewer when the batch's longest A has fewer
 *                 512-column strips or the shared memory holds fewer),
 *                 0 = no teams.  A team's warps take the strips of one pair
 *                 couple round robin (forward pass, then the reverse pass
 *                 for start coordinates), so a long pair finishes up to that
 *                 many times sooner; the cost model sends a pair there when
 *                 its one-warp latency exceeds half of the batch's modelled
 *                 time and a team finishes it sooner
 *   "chunks"      ipuma_gpu_compare(_packed) only: 0 = split large batches into up
 *                 to 8 chunks whose uploads overlap the alignment of the
 *                 previous chunks (default), 1 = upload everything first,
 *                 n = exactly n chunks (at most 8) */
int ipuma_gpu_set_option(ipuma_engine* e, const char* name, int64_t value);

/* Runs one batch in the reference wire format and waits for it.
 *   inputs  : n_inputs int32 = Seqs (tiles_used x ceil(bufsize/4) words of
 *             uint8 codes) || Meta (tiles_used x max_batches x {a_len, a_off,
 *             b_len, b_off}), as written by SWAlgorithm::prepare_remote
 *   results : n_results = 3 * tiles_used * max_batches int32 =
 *             scores || a_ranges || b_ranges, indexed tile*max_batches+slot;
 *             ranges pack start | end << 16 (uint16 halves). */
int ipuma_gpu_run_buffer(ipuma_engine* e, const int32_t* inputs, size_t n_inputs, int32_t* results,
                         size_t n_results);
/* Asynchronous form: the buffers must stay valid until ipuma_gpu_join.
 * Returns once the work is enqueued.  Jobs alternate between two device
 * buffer sets and streams, so one job's upload and result copy overlap the
 * previous job's kernels; only the tiles up to the last one with a
 * non-zero Meta word are uploaded.  Pageable `results` receive the job's
 * results through pinned staging, copied out by the join. */
int ipuma_gpu_submit_buffer(ipuma_engine* e, const int32_t* inputs, size_t n_inputs,
                            int32_t* results, size_t n_results, uint64_t* job);
/* *done = 1 once the job's results are in place (results are only
 * guaranteed after ipuma_gpu_join). */
int ipuma_gpu_poll(ipuma_engine* e, uint64_t job, int32_t* done);
/* Waits for a job (bounded by timeout_ms; < 0 waits without limit).  A job
 * is joined once; jobs may be joined in any order, from any thread. */
int ipuma_gpu_join(ipuma_engine* e, uint64_t job, int64_t timeout_ms);
/* ipuma_gpu_join that also returns the job's own statistics (kernel_ms =
 * its kernels, total_ms = upload + kernels + result copy), whatever other
 * jobs ran or were joined meanwhile.  `out` may be null. */
int ipuma_gpu_join_stats(ipuma_engine* e, uint64_t job, int64_t timeout_ms, ipuma_stats* out);

/* Aligns n pairs from host memory; results in input order.  Large batches
 * are split into chunks of consecutive pairs: each chunk uploads the byte
 * ranges of `codes` its pairs read (the span of its A offsets and the span
 * of its B offsets) while earlier chunks compute, so the copy overlaps the
 * kernels when sequences are stored in pair order. */
int ipuma_gpu_compare(ipuma_engine* e, const uint8_t* codes, size_t n_codes,
                      const ipuma_pair* pairs, int32_t n, int32_t* score, int32_t* arange,
                      int32_t* brange);
/* ipuma_gpu_compare with packed codes (ipuma_pack_codes):
 *   bits = 5: amino acids (or any alphabet of at most 32 codes);
 *   bits = 4: alphabets of at most 16 codes (nucleic acids with IUPAC);
 *   bits = 2: A, T, C, G only (nucleic acids, codes 1..4).
 * n_codes, offsets and lengths count residues.  The codes travel and stay
 * packed: the kernels read the bit stream themselves, so the upload and
 * the device copy are bits/8 of the one-byte form. */
int ipuma_gpu_compare_packed(ipuma_engine* e, const uint8_t* packed, size_t n_codes, int32_t bits,
                             const ipuma_pair* pairs, int32_t n, int32_t* score, int32_t* arange,
                             int32_t* brange);
/* Same with every buffer in device memory, enqueued on `stream`
 * (cudaStream_t, NULL = the engine's stream); max_a_len / max_b_len bound
 * the pair lengths.  Every descriptor is checked on the device before any
 * code is read: a length past those bounds gives IPUMA_ERR_TOO_LONG, a
 * negative field or a sequence reaching past the n_codes residues of
 * d_codes IPUMA_ERR_INVALID_ARG; those pairs get a zero result. */
int ipuma_gpu_compare_device(ipuma_engine* e, const uint8_t* d_codes, size_t n_codes,
                             const ipuma_pair* d_pairs, int32_t n, int32_t max_a_len,
                             int32_t max_b_len, int32_t* d_score, int32_t* d_arange,
                             int32_t* d_brange, void* stream);
/* ipuma_gpu_compare_device on packed codes (ipuma_pack_codes layout, bits =
 * 2, 4 or 5) that the kernels read directly.  d_packed starts 4-byte
 * aligned and is readable for ceil(n_codes * bits / 8) bytes rounded up to
 * a multiple of 4, plus 4 more bytes (the word after the last residue's). */
int ipuma_gpu_compare_device_packed(ipuma_engine* e, const uint8_t* d_packed, size_t n_codes, int32_t bits,
                                    const ipuma_pair* d_pairs, int32_t n, int32_t max_a_len,
                                    int32_t max_b_len, int32_t* d_score, int32_t* d_arange,
                                    int32_t* d_brange, void* stream);

/* Grows every device buffer that ipuma_gpu_compare_device needs for up to
 * n pairs with |A| <= max_a_len and |B| <= max_b_len, so that such calls
 * allocate (and synchronise the device) no more -- for serving loops and
 * before a stream capture.  No counterpart in the reference. */
int ipuma_gpu_reserve(ipuma_engine* e, int32_t n, int32_t max_a_len, int32_t max_b_len);

/* Wire-buffer batch with inputs and results already in device memory,
 * enqueued on `stream` (NULL = the engine's stream); the call returns once
 * the batch has finished.  Sizes as for ipuma_gpu_run_buffer; the Meta
 * section is validated on the device. */
int ipuma_gpu_run_buffer_device(ipuma_engine* e, const int32_t* d_inputs, size_t n_inputs,
                                int32_t* d_results, size_t n_results, void* stream);

int ipuma_gpu_last_stats(ipuma_engine* e, ipuma_stats* out);

/* Autotuner: measures, for this engine's GPU and alphabet, the rates of the
 * kernel classes that the cost-binned scheduler chooses between (lanes per
 * group, columns per lane), or loads them from `cache_path` (a file of
 * tab-separated lines; NULL = the IPUMA_TUNE_CACHE environment variable or
 * none).  Runs once per process and key; with option "autotune" = 1 (the
 * default) the first batched call runs it implicitly. */
int ipuma_gpu_autotune(ipuma_engine* e, const char* cache_path);
/* Writes the rates in use as JSON text into buf. */
int ipuma_gpu_tuning(ipuma_engine* e, char* buf, size_t cap);

/* Allocation-free alignment, for callers that cannot call cudaMalloc: host
 * programs whose own memory pool owns all device memory (for example a
 * framework's caching allocator that reserved the GPU) and paths that
 * cannot afford the device-wide synchronisation cudaMalloc/cudaFree imply.
 * No counterpart in the reference.  Aligns n pairs on the current device
 * with exact 32-bit lanes; codes (n_codes residues), pairs and the three
 * result arrays are device memory owned by the caller; results as
 * ipuma_gpu_compare.  Nothing is allocated: the kernel's strip-boundary
 * scratch is a 16 MiB file-scope device array that every GPU loading the
 * library holds until exit.  Limits: max_b_len (an upper bound of every
 * b_len, checked on the device) at most 65535, every a_len at most 65535;
 * gap_init + gap_extend < 0 and gap_extend <= 0.  Pairs are checked on the
 * device before any code is read: a length beyond those limits gives
 * IPUMA_ERR_TOO_LONG, a negative field or a sequence past n_codes
 * IPUMA_ERR_INVALID_ARG (those pairs get a zero result).  The first call on
 * a device looks up the array's device address, so make it before any
 * stream capture.  All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller.  Blocks until the batch
 * is done; errors through ipuma_last_error(). */
int ipuma_gpu_compare_noalloc(const ipuma_sw_config* sw, int32_t forward_only, const uint8_t* d_codes,
                              size_t n_codes, const ipuma_pair* d_pairs, int32_t n, int32_t max_b_len,
                              int32_t* d_score, int32_t* d_arange, int32_t* d_brange, void* stream);

/* ---- serving loop ------------------------------------------------------- */
/* Continuous batching of alignment requests on one GPU: requests queue on
 * the host; `slots` workers (one engine and CUDA stream each) take whatever
 * is queued for one scoring configuration into a device batch, so requests
 * that arrive while others run join the next batch and batches of
 * different slots overlap on the device.  Batches get their device memory
 * from a pool allocated when the server starts (admission by free HBM: a
 * batch waits until the pool has room).  No counterpart API in the
 * reference; it generalises the pipelined use of
 * async_submit_prepared_remote_compare / blocking_join (ipusw). */
typedef struct ipuma_server_config {
  int32_t n_scorings;              /* scoring configurations; requests pick one by index */
  const ipuma_sw_config* scorings;
  int32_t forward_only;            /* 1: no reverse pass (start coordinates 0) */
  int32_t slots;                   /* concurrent device batches; 0 = 4 */
  int64_t pool_bytes;              /* device pool; 0 = a quarter of the free memory */
  int32_t max_batch_pairs;         /* pairs per device batch; 0 = 262144 */
  int32_t device;
  int32_t one_request_per_batch;   /* 1: no coalescing (each batch = one request or
                                      part of one), the per-request baseline */
  int64_t max_batch_cells;         /* cells per device batch (latency bound); 0 = 2e10 */
  int32_t reserve_b_len;           /* |B| the engines' buffers are sized for at start;
                                      0 = 2048 (longer pairs grow them on demand) */
} ipuma_server_config;

typedef struct ipuma_server_stats {
  int64_t submitted, completed, queued, batches, pairs, cells;
  int64_t max_batch_pairs;         /* largest batch formed */
  int64_t pool_bytes, pool_used, max_pool_used;
  double busy_ms;                  /* summed slot time with a batch in flight */
} ipuma_server_stats;

typedef struct ipuma_server ipuma_server;

int ipuma_server_create(const ipuma_server_config* cfg, ipuma_server** out);
/* Queues one request (the buffers are copied before the call returns).
 * IPUMA_ERR_CLOSED after ipuma_server_destroy began; IPUMA_ERR_NO_MEMORY
 * when one of its pairs cannot fit the device pool. */
int ipuma_server_submit(ipuma_server* s, int32_t kind, const uint8_t* codes, size_t n_codes,
                        const ipuma_pair* pairs, int32_t n, uint64_t* req);
/* Uploads a code array once into device memory that the server keeps
 * until it is destroyed (outside the batch pool; IPUMA_ERR_NO_MEMORY when
 * the device has no room) and returns its set id. */
int ipuma_server_add_sequences(ipuma_server* s, const uint8_t* codes, size_t n_codes, int32_t* set_id);
/* Queues a request whose pairs index a resident set (offsets into the
 * codes given to ipuma_server_add_sequences): only the pair descriptors
 * are copied and staged. */
int ipuma_server_submit_resident(ipuma_server* s, int32_t kind, int32_t set_id, const ipuma_pair* pairs,
                                 int32_t n, uint64_t* req);
int ipuma_server_poll(ipuma_server* s, uint64_t req, int32_t* done);
/* Waits for a request (timeout_ms < 0: no limit) and copies its results
 * (in pair order) and its latency from submission to completion.  A
 * request id is released by a successful or failed wait. */
int ipuma_server_wait(ipuma_server* s, uint64_t req, int64_t timeout_ms, int32_t* score, int32_t* arange,
                      int32_t* brange, double* latency_ms);
int ipuma_server_get_stats(ipuma_server* s, ipuma_server_stats* out);
/* Stops accepting requests (submit returns IPUMA_ERR_CLOSED); queued and
 * running work still completes and can be waited for. */
int ipuma_server_close(ipuma_server* s);
/* Closes, finishes queued and running work, then releases the server. */
void ipuma_server_destroy(ipuma_server* s);

/* Measures, on `device`, the issue rate of the s16x2 instruction mix of one
 * cell update (3 add, 2 viaddmax, 1 vimax3.relu, 1 max) in lane-ops per
 * second: the peak against which the kernels' roofline fraction is taken. */
int ipuma_measure_int_peak(int32_t device, double* lane_ops_per_s);

#ifdef __cplusplus
}
#endif
#endif /* IPUMA_B200_H */
