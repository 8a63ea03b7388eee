/*
 * sa_b200.h -- C ABI of the B200 banded pair-HMM engine (signalAlign's signal-to-reference
 * posterior alignment).  Plain C types only: pointers, sizes, int64/double.  All entry points
 * return an sa_status (0 = SA_OK) and never abort the process.
 *
 * Each declaration names the signalAlign routine it replaces (file:line in the signalAlign tree).
 */
#ifndef SA_B200_H_
#define SA_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference aborts through st_errAbort / assert instead) ---- */
typedef enum {
    SA_OK = 0,
    SA_E_ARG = 1,            /* bad argument (NULL pointer, negative length, bad parameters)            */
    SA_E_ALPHABET = 2,       /* k-mer character outside the model alphabet (kmer_to_word exit,
                                nanopore_hdp.c:375-388)                                                  */
    SA_E_ANCHORS = 3,        /* anchors not strictly increasing / outside the matrix (band_construct
                                asserts, pairwiseAligner.c:160-167; getSplitPoints asserts :1743-1746)  */
    SA_E_NOMEM = 4,          /* host or device allocation failed                                        */
    SA_E_CUDA = 5,           /* CUDA runtime error                                                      */
    SA_E_OUTPUT = 6,         /* pair output buffer too small (re-run with a larger capacity)            */
    SA_E_UNSUPPORTED = 7,    /* combination this engine does not run (e.g. 5-state machines)            */
    SA_E_FILE = 8,           /* .model / .nhdp file missing or malformed (stateMachine.c:1339-1426,
                                hdp.c:3047-3316)                                                         */
    SA_E_TIMEOUT = 9,        /* a bounded device-side wait gave up                                      */
    SA_E_DEVICE = 10,        /* device-side consistency check failed                                    */
    SA_E_CAPACITY = 11       /* request larger than a fixed capacity of the entry point                 */
} sa_status;

/* ---- state machine (StateMachine / StateMachine3 / StateMachine3_HDP, inc/stateMachine.h:76-182) ---- */
typedef enum {
    SA_THREE_STATE = 2,      /* StateMachineType threeState (inc/stateMachine.h:30)                      */
    SA_THREE_STATE_HDP = 7   /* StateMachineType threeStateHdp (inc/stateMachine.h:35)                   */
} sa_machine_type;

typedef enum {
    SA_EMIT_PLAIN = 0,       /* emissions_signal_strawManGetKmerEventMatchProb (stateMachine.c:547-589),
                                used by getStateMachine3 (stateMachine.c:1645-1653)                      */
    SA_EMIT_DESCALED = 1,    /* ..._strawManGetKmerEventMatchProbWithDescaling (stateMachine.c:498-545),
                                used by getStateMachine3_descaled (stateMachine.c:1627-1643)             */
    SA_EMIT_HDP = 2          /* emissions_signal_getHdpKmerDensity (stateMachine.c:468-495), used by
                                getHdpStateMachine (stateMachine.c:1655-1669)                            */
} sa_emission;

/* transition slots in log space, StateMachine3 field order (inc/stateMachine.h:153-163) */
enum {
    SA_T_MATCH_CONTINUE = 0, SA_T_MATCH_FROM_GAP_X, SA_T_MATCH_FROM_GAP_Y, SA_T_GAP_OPEN_X,
    SA_T_GAP_OPEN_Y, SA_T_GAP_EXTEND_X, SA_T_GAP_EXTEND_Y, SA_T_GAP_SWITCH_TO_X, SA_T_GAP_SWITCH_TO_Y,
    SA_N_TRANSITIONS
};

/* DegenerateType (inc/pairwiseAligner.h:50-56): which bases an 'X' in the reference may be */
typedef enum {
    SA_CYTOSINE_METHYLATION2 = 0,   /* "CE"   */
    SA_CYTOSINE_METHYLATION3 = 1,   /* "CEO"  */
    SA_ADENOSINE_METHYLATION = 2,   /* "AI"   */
    SA_CANONICAL_VARIANTS = 3       /* "ACGT" */
} sa_degenerate;

typedef struct sa_state_machine sa_state_machine;   /* opaque; its tables live on the device */

/* stateMachine3_loadFromFile (stateMachine.c:1328-1426) + getStateMachine3 / getStateMachine3_descaled /
 * getHdpStateMachine (stateMachine.c:1627-1669).  For SA_THREE_STATE_HDP, nhdp_file is read as by
 * deserialize_nhdp (nanopore_hdp.c:1071-1098); set_hdp_expected_values applies
 * stateMachine3_setModelToHdpExpectedValues (stateMachine.c:1163-1192), as signalMachine does
 * (signalMachine.c:709-711).  `device` is the CUDA device that holds the tables. */
sa_status sa_stateMachine_loadFromFile(const char *model_file, sa_machine_type type, sa_emission emission,
                                       const char *nhdp_file, int32_t set_hdp_expected_values, int32_t device,
                                       sa_state_machine **out);

/* Same state machine from in-memory tables.  match/gap_y: n_kmers x 5 doubles (level_mean, level_sd,
 * noise_mean, noise_sd, noise_lambda) in k-mer-id order; gap_y's level_sd already multiplied by
 * EXTRA_EVENT_NOISE_MULTIPLIER as the loader does (stateMachine.c:1418-1420); gap_x: n_kmers log
 * probabilities (log 0.1 in the reference, stateMachine.c:1472-1474). */
sa_status sa_stateMachine_fromTables(sa_machine_type type, sa_emission emission, const char *alphabet,
                                     int32_t alphabet_size, int32_t kmer_length,
                                     const double transitions[SA_N_TRANSITIONS], const double *match,
                                     const double *gap_y, const double *gap_x, int32_t device,
                                     sa_state_machine **out);

/* HDP posterior-predictive tables (dir_proc_density, hdp.c:2583-2607): a uniform grid
 * linspace(grid_start, grid_stop, grid_length) (hdp_math_utils.c:497-509), n_rows rows of density
 * and knot slopes, and per k-mer the row of its nearest observed ancestor (-1: none). */
sa_status sa_stateMachine_setHdp(sa_state_machine *sm, double grid_start, double grid_stop,
                                 int64_t grid_length, int64_t n_rows, const double *density,
                                 const double *slope, const int64_t *kmer_row);

/* scale/shift/var of the StateMachine (inc/stateMachine.h:82-84, set at stateMachine.c:1633-1635). */
sa_status sa_stateMachine_setScaling(sa_state_machine *sm, double scale, double shift, double var);

/* emissions_signal_scaleModel (stateMachine.c:630-668) and emissions_signal_scaleNoise
 * (stateMachine.c:607-628), applied to the state machine's tables in place. */
sa_status sa_stateMachine_scaleModel(sa_state_machine *sm, double scale, double shift, double var,
                                     double scale_sd, double var_sd);
sa_status sa_stateMachine_scaleNoise(sa_state_machine *sm, double scale_sd, double var_sd);

/* model facts and the interned, process-lifetime path k-mer string of a k-mer id (the reference puts
 * the path's char* into element 3 of each aligned pair, pairwiseAligner.c:1239-1241). */
int32_t sa_stateMachine_kmerLength(const sa_state_machine *sm);
int64_t sa_stateMachine_numberOfKmers(const sa_state_machine *sm);
const char *sa_stateMachine_kmerString(const sa_state_machine *sm, int64_t kmer_id);

/* kmer_id (nanopore_hdp.c:388-393) over the state machine's sorted alphabet; -1 if a character is
 * outside it. */
int64_t sa_stateMachine_kmerId(const sa_state_machine *sm, const char *kmer);

/* the model's tables back on the host (for checking a load): match/gap_y n x 5, gap_x n, t[9] */
sa_status sa_stateMachine_getTables(const sa_state_machine *sm, double *match, double *gap_y, double *gap_x,
                                    double *transitions);

/* the machine's HDP tables back on the host (for checking a .nhdp load, as deserialize_nhdp would
 * hold them, nanopore_hdp.c:1071-1098): the grid, n_rows rows of posterior-predictive density and
 * knot slopes, and per k-mer its row (-1: no observed ancestor).  Arrays may be NULL: a first call
 * with NULL arrays returns the sizes.  SA_E_UNSUPPORTED for a machine without HDP tables. */
sa_status sa_stateMachine_getHdpTables(const sa_state_machine *sm, int64_t *grid_length, int64_t *n_rows,
                                       double *grid, double *density, double *slope, int64_t *kmer_row);

void sa_stateMachine_destruct(sa_state_machine *sm);

/* ---- alignment parameters (PairwiseAlignmentParameters, inc/pairwiseAligner.h:123-134) ---- */
typedef struct {
    double threshold;                     /* posterior threshold, default 0.01 */
    int64_t min_diags_between_traceback;  /* default 1000 */
    int64_t traceback_diagonals;          /* default 40   */
    int64_t diagonal_expansion;           /* default 20 in the library, 50 in signalMachine */
    int64_t constraint_diagonal_trim;     /* default 14 (anchor preparation only) */
    int64_t split_matrix_bigger_than_this;/* default 3000*3000 */
} sa_params;

/* pairwiseAlignmentBandingParameters_construct (pairwiseAligner.c:1843-1856) */
void sa_params_default(sa_params *p);

/* ---- one aligned pair: stIntTuple(4) of getAlignedPairsUsingAnchors (pairwiseAligner.c:1237-1241) ---- */
typedef struct {
    int64_t score;   /* floor(posterior * 10^7)  (PAIR_ALIGNMENT_PROB_1, inc/pairwiseAligner.h:27) */
    int64_t x;       /* reference k-mer index */
    int64_t y;       /* event index */
    int64_t kmer;    /* path k-mer id; sa_stateMachine_kmerString gives its string */
} sa_aligned_pair;

/* ---- band geometry and split points (host, bit-exact with the reference) ---- */

/* band_construct (pairwiseAligner.c:131-182): xmyL/xmyR of every anti-diagonal xay = 0..lX+lY.
 * anchors: n_anchors (x, y) pairs in k-mer / event coordinates, strictly increasing. */
sa_status sa_band_construct(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t expansion,
                            int64_t *xmy_l, int64_t *xmy_r);

/* getSplitPoints (pairwiseAligner.c:1730-1757): writes up to max_regions (x1, y1, x2, y2) tuples and
 * their count. */
sa_status sa_getSplitPoints(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY,
                            int64_t split_matrix_bigger_than_this, int32_t ragged_left, int32_t ragged_right,
                            int64_t *regions, int64_t max_regions, int64_t *n_regions);

/* ---- plain FP64 form: one read per launch ---- */

/* getAlignedPairsUsingAnchors(sM, sX, sY, anchorPairs, p, diagonalCalculationPosteriorMatchProbs,
 * raggedLeft, raggedRight) (pairwiseAligner.c:1871-1899), which splits at large anchor gaps
 * (:1773-1837) and runs getPosteriorProbsWithBanding (:1282-1420) on each region.
 *   reference: nucleotide string of reference_length chars (lX = reference_length - (k-1) k-mers),
 *              'X' expands to the bases of `degenerate` (hdCell_construct, :605-650);
 *   events: n_events x 4 doubles (mean, noise, duration, start; NB_EVENT_PARAMS, inc/nanopore.h:4);
 *   anchors: n_anchors (x, y) pairs.
 * The pairs come back in the reference's emission order.  *pairs is allocated with malloc; free it
 * with sa_free_pairs.  Optional: log_likelihood receives the total probability of the last region's
 * final refresh (the normaliser of its last posteriors). */
sa_status sa_getAlignedPairsUsingAnchors(const sa_state_machine *sm, const char *reference,
                                         int64_t reference_length, sa_degenerate degenerate,
                                         const double *events, int64_t n_events, const int64_t *anchors,
                                         int64_t n_anchors, const sa_params *p, int32_t ragged_left,
                                         int32_t ragged_right, sa_aligned_pair **pairs, int64_t *n_pairs,
                                         double *log_likelihood);

void sa_free_pairs(sa_aligned_pair *pairs);

/* ---- batched FP32 form: many reads, one persistent launch ---- */

/* One read of a batch: the inputs of signalMachine's performSignalAlignment (signalMachine.c:333-354)
 * after anchor remapping, plus the read's NanoporeReadAdjustmentParameters (inc/nanopore.h:11-19). */
typedef struct {
    const sa_state_machine *sm;   /* model; emission kind and tables come from it */
    const char *reference;        /* nucleotide string */
    int64_t reference_length;
    const double *events;         /* n_events x 4 doubles */
    int64_t n_events;
    const int64_t *anchors;       /* n_anchors x (x, y) */
    int64_t n_anchors;
    double scale, shift, var;     /* used by SA_EMIT_DESCALED / SA_EMIT_HDP (descaleEventMean_JordanStyle) */
    int32_t ragged_left, ragged_right;
    int32_t degenerate;           /* sa_degenerate */
    int32_t pad;
} sa_read;

typedef struct sa_batch sa_batch;   /* opaque: packed inputs, device buffers, results */

/* Host-side planning of a batch: band geometry, traceback windows, k-mer ids, packing; allocates the
 * batch's device buffers on the state machines' device.  The reads' arrays are copied; the caller
 * may free them after this returns. */
sa_status sa_batch_create(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch **out);

/* host -> device copy of the packed inputs on `stream` (a cudaStream_t, NULL = default stream) */
sa_status sa_batch_upload(sa_batch *b, void *stream);

/* the alignment itself on `stream`: one persistent FP32 launch over all regions (inputs resident) */
sa_status sa_batch_run(sa_batch *b, void *stream);

/* device -> host copy of pair counts, pairs and per-read status; synchronises `stream` */
sa_status sa_batch_download(sa_batch *b, void *stream);

/* all of the above in one call */
sa_status sa_align_batch(const sa_read *reads, int64_t n_reads, const sa_params *p, void *stream,
                         sa_batch **out);

/* results after download: per read status, pair count and pairs (reference emission order) */
sa_status sa_batch_read_status(const sa_batch *b, int64_t read);
int64_t sa_batch_pair_count(const sa_batch *b, int64_t read);
const sa_aligned_pair *sa_batch_pairs(const sa_batch *b, int64_t read);
/* the total probability of each read's last refresh (log-likelihood of its final window) */
double sa_batch_log_likelihood(const sa_batch *b, int64_t read);
/* batch facts: DP cells (sum of band widths over all regions) and regions */
int64_t sa_batch_cells(const sa_batch *b);
/* bytes the batch moves host->device on upload and device->host on download (after a download) */
sa_status sa_batch_transfer_bytes(const sa_batch *b, int64_t *h2d, int64_t *d2h);
int64_t sa_batch_regions(const sa_batch *b);
/* device time (CUDA events) of the last sa_batch_run's three kernels: per-cell emissions, the
 * forward / traceback-window worker, the pair gather.  Waits for them.  SA_E_ARG if the batch has
 * not run (no counterpart in signalAlign: a diagnostic of this engine) */
sa_status sa_batch_kernel_ms(const sa_batch *b, double *emission_ms, double *worker_ms, double *gather_ms);
/* ---- launch configuration of the batched FP32 kernels, and its tuner (no counterpart in signalAlign,
 * which has no GPU code) ----
 * Per device (by name) and band-width class (1: bands up to 128 cells, 2: up to 256, 4: up to 512)
 * one configuration; a device without one uses the defaults below, measured on B200. */
typedef struct {
    int32_t ctas_per_sm;           /* worker CTAs per SM (at most the kernel's occupancy; default 2) */
    int32_t grid_per_region;       /* worker grid at most this many CTAs per region (default 3) */
    int32_t warp_windows;          /* class 1: a traceback window per warp (1, default) or per CTA (0) */
    int32_t emission_ctas_per_sm;  /* emission kernel grid, CTAs per SM (default 16) */
} sa_launch_config;

/* the configuration sa_batch_run uses on `device` for a width class */
sa_status sa_getLaunchConfig(int32_t device, int32_t width_class, sa_launch_config *cfg);
/* sets it for every device with the same name as `device` (values out of range: SA_E_ARG) */
sa_status sa_setLaunchConfig(int32_t device, int32_t width_class, const sa_launch_config *cfg);
/* Times every candidate configuration on a created and uploaded batch (`repeats` runs each after
 * one untimed run, device time of its kernels by CUDA events), sets the fastest for the batch's
 * device and width class, and returns it with its mean time; *n_tried counts the candidates.
 * The batch's results are those of its last run. */
sa_status sa_tuneLaunchConfig(sa_batch *b, void *stream, int32_t repeats, sa_launch_config *best, double *best_ms,
                              int32_t *n_tried);
/* Reads configurations from a text file, one per line: device name, width class and the four
 * fields, tab-separated (lines starting with '#' are comments); they apply to devices of that name.
 * A missing file is SA_E_FILE. */
sa_status sa_loadLaunchConfigs(const char *path);

/* Bound, in SM clock cycles, of every device-side wait of the batch's worker kernel (a warp waiting
 * for a traceback window to be published).  Default 2e10 (about 10 s), far beyond any forward sweep.
 * A wait that runs out sets the batch's error flag: every other waiter leaves, the kernel ends
 * normally, and every read of the batch reports SA_E_TIMEOUT.  No counterpart in signalAlign (its
 * CPU code never waits); a diagnostic of this engine's bounded waits. */
sa_status sa_batch_set_wait_limit(sa_batch *b, int64_t cycles);

/* ---- forward segments (no counterpart in signalAlign, whose forward sweep runs once per region) ----
 * A region's forward sweep is sequential over its anti-diagonals, so the longest read of a batch
 * bounds the batch.  Both forms (the batched FP32 form and the plain FP64 form behind
 * sa_getAlignedPairsUsingAnchors and a batch's X reads; not the expectations calls) cut it at
 * traceback-window starts into segments that run at the same time on different CTAs.  Each segment after the first sweeps max(warmup_diags, 10 x the
 * region's widest anti-diagonal) anti-diagonals before its own from a flat start; its values then
 * equal the true ones minus one constant (the recursion depends only on differences of log values,
 * and the start's influence dies out within a few band widths).  Where two segments meet, the kernel checks that on two
 * anti-diagonals (FP32: every cell within 2e-5 + 1e-6 x its distance below the anti-diagonal's
 * maximum; FP64: 1e-9 + 1e-11 x that distance);
 * posteriors do not depend on the constant, and the log-likelihood adds it back.  A read whose
 * check disagrees is re-run unsegmented at download, so results never depend on it.
 * segment_diags: < 0 keeps every region whole; > 0 caps a segment's sweep (warm-up included);
 * 0 (default) picks twice the batch's forward anti-diagonals per worker CTA, at least 4096 (a large
 * batch, bound by its total work, then keeps nearly every region whole; a small one splits).
 * warmup_diags: default 1024, at least 64.  Applies to batches created afterwards. */
sa_status sa_setSegmentPolicy(int32_t segment_diags, int32_t warmup_diags);
sa_status sa_getSegmentPolicy(int32_t *segment_diags, int32_t *warmup_diags);
/* The forward segments the batched form would plan for one read (host only, no device): per
 * segment 6 int64 (region, first anti-diagonal b (exclusive unless 0), last anti-diagonal, warm-up
 * anti-diagonals, region-relative index of the first window it publishes, region's widest
 * anti-diagonal), for an explicit cap segment_diags > 0 (or < 0: regions whole).  Ragged ends as
 * signalMachine passes them.  SA_E_OUTPUT with *n_segments set when capacity is too small. */
sa_status sa_planForwardSegments(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY,
                                 const sa_params *p, int32_t segment_diags, int32_t warmup_diags, int64_t *out,
                                 int64_t capacity, int64_t *n_segments);
/* segments and stitches of a batch (both forms); after a download, reads (FP32 form) and regions
 * (plain form) re-run unsegmented, and the largest deviation from the constant over the FP32 form's
 * agreeing stitches */
sa_status sa_batch_segment_info(const sa_batch *b, int64_t *n_segments, int64_t *n_stitches, int64_t *n_redone,
                                double *max_spread);
/* scale of the stitch tolerance for the batch's next runs (default 1; a negative scale makes every
 * stitch disagree, which exercises the unsegmented re-run) */
sa_status sa_batch_set_stitch_tolerance(sa_batch *b, double scale);
void sa_batch_destroy(sa_batch *b);

/* ---- batched FP32 form without device allocation (no counterpart in signalAlign) ---- */

/* Size of the one static device array behind sa_align_batch_noalloc, per device: 64 MiB, room for
 * about 3 million band cells with their inputs and pair output (e.g. ten reads of 1 kb reference
 * and 1.5k events at diagonal expansion 50). */
#define SA_NOALLOC_SCRATCH_BYTES (64ll << 20)

/* sa_align_batch for callers that must not allocate device memory.  Such callers exist: a process
 * whose framework already holds almost all of the GPU's memory in its own pool (a caching allocator,
 * a serving engine that reserved its arena at start-up), where cudaMalloc fails or makes the
 * framework give memory back; and latency-bound loops, where cudaMalloc / cudaFree can synchronise
 * the whole device and stall every other stream.  This call runs the same batched FP32 kernel as
 * sa_align_batch, with every device buffer (packed inputs, forward store, counters, pair output)
 * carved from one file-scope device array of SA_NOALLOC_SCRATCH_BYTES; it calls no cudaMalloc,
 * cudaFree or other allocating routine.
 *   - Each read's state machine must already hold current device tables (they are written by the
 *     first allocating call that uses the machine after it was loaded or changed: sa_align_batch,
 *     sa_batch_create, sa_getAlignedPairsUsingAnchors); otherwise SA_E_ARG.
 *   - A batch that needs more than SA_NOALLOC_SCRATCH_BYTES is rejected with SA_E_CAPACITY before
 *     any device work; *scratch_bytes (optional) receives the bytes the batch needs in every case.
 *   - Reads only the plain FP64 form runs (references with 'X' positions; machines whose gap-Y
 *     table has its own level means or noise, as after sa_stateMachine_loadExpectations with an
 *     event model) get read status SA_E_UNSUPPORTED; the others are aligned.
 *   - What must be zero when the kernel starts (the region queue counter, per-read status words and
 *     per-region pair counts) is cleared by the call itself on `stream` before every launch; every
 *     other byte the kernel reads is written earlier in the same call.
 *   - The first call on a device looks the array's address up (cudaGetSymbolAddress, which can load
 *     the library's device code on that device): make one call on each device during set-up, before
 *     any stream capture begins.  With lazy module loading that first call is also when the device
 *     reserves the array's SA_NOALLOC_SCRATCH_BYTES, so make it before the host framework reserves
 *     its own memory pool; if the device has no room left by then the call returns SA_E_CUDA.
 *   - All calls on a device share the array, so two calls whose device work overlapped would
 *     overwrite each other's data.  The call is synchronous (it returns after `stream` drained) and
 *     holds a per-device lock for its whole duration, so calls from several host threads run one
 *     after another.
 * Results: read r's pairs are pairs[pair_offsets[r] .. pair_offsets[r + 1]) (reference emission
 * order); pair_offsets has n_reads + 1 entries; read_status n_reads entries (as
 * sa_batch_read_status); log_likelihood n_reads entries or NULL.  If the pairs exceed pair_capacity
 * the call returns SA_E_OUTPUT with pair_offsets filled (pair_offsets[n_reads] is the capacity
 * needed) and writes no pair. */
sa_status sa_align_batch_noalloc(const sa_read *reads, int64_t n_reads, const sa_params *p, void *stream,
                                 sa_aligned_pair *pairs, int64_t pair_capacity, int64_t *pair_offsets,
                                 int32_t *read_status, double *log_likelihood, int64_t *scratch_bytes);

/* ---- serving: reads aligned as they arrive, with continuous batching ----
 * No counterpart in signalAlign, which aligns one read per process (scripts/runSignalAlign.py:176-224).
 * A dispatcher thread admits waiting reads into a new micro-batch whenever a stream is free and the
 * band cells in flight (estimated as (reference_length + n_events + 1) x (diagonal_expansion + 1)
 * per read) stay within max_inflight_cells; each micro-batch runs on its own stream, beside the ones
 * already on the device.  A read finishes as soon as its own traceback windows have: the worker
 * kernel publishes it to mapped host memory and its pairs are copied while the kernel runs on.
 * A read's result does not depend on which reads share its micro-batch. */
typedef struct sa_server sa_server;
sa_status sa_server_create(int32_t device, int64_t max_inflight_cells, int32_t max_batches, sa_server **out);
/* queue one read (its arrays are copied); *ticket identifies it */
sa_status sa_server_submit(sa_server *s, const sa_read *read, const sa_params *p, int64_t *ticket);
/* block until the read is done or timeout_ms passed (SA_E_TIMEOUT) */
sa_status sa_server_wait(sa_server *s, int64_t ticket, double timeout_ms);
/* a finished read: its status, pairs (owned by the server until sa_server_release), log-likelihood
 * and latency from submission to completion in milliseconds (either may be NULL) */
sa_status sa_server_result(sa_server *s, int64_t ticket, int32_t *status, const sa_aligned_pair **pairs,
                           int64_t *n_pairs, double *log_likelihood, double *latency_ms);
sa_status sa_server_release(sa_server *s, int64_t ticket);
/* finishes the queued reads, then stops the dispatcher */
void sa_server_destroy(sa_server *s);
typedef struct sa_server_counters {
    int64_t reads_early;          /* reads finished when the kernel published them */
    int64_t reads_at_batch_end;   /* reads finished with their micro-batch (plain form, errors) */
    int64_t batches;              /* micro-batches finished */
    double admit_ms;              /* dispatcher time planning, uploading and launching micro-batches */
    double fetch_ms;              /* dispatcher time copying published reads' pairs */
    double finish_ms;             /* dispatcher time finishing micro-batches */
    double plan_ms;               /* the planning part of admit_ms (sa_batch_create) */
    double upload_ms;             /* the upload part of admit_ms (sa_batch_upload) */
} sa_server_counters;
sa_status sa_server_stats(sa_server *s, sa_server_counters *out);
/* a finished read's wait: from submission to the start of its micro-batch's admission, and from
 * there to its kernels' launch (planning and upload); both 0 for a read that was never launched.
 * The rest of its latency is the kernels and the copy of its pairs. */
sa_status sa_server_read_timing(sa_server *s, int64_t ticket, double *queue_ms, double *launch_ms);
/* per finished micro-batch, in finishing order, three doubles: device time of its start (before its
 * emission kernel) and of its worker kernel's end, in ms from the server's creation, and its read
 * count (0, 0 when the batch was not timed); min(capacity, n) triples are written */
sa_status sa_server_batch_log(sa_server *s, double *out, int64_t capacity, int64_t *n_batches);

/* ---- EM expectations: the same path with the expectation epilogue (pairwiseAligner.c:1983-2003) ---- */

/* the accumulators of a continuous pair HMM (continuousPairHmm_construct, continuousHmm.c:84-141);
 * the caller owns the arrays and initialises them (transitions and posteriors to the pseudocounts,
 * the rest to zero, as hmmContinuous_getExpectationsHmm does); calls accumulate into them */
typedef struct {
    double likelihood;            /* += the total probability of every posterior anti-diagonal */
    double transitions[9];        /* from * 3 + to; states: 0 match, 1 skip (gap-X), 2 extra event (gap-Y) */
    double *event_expectations;   /* n_kmers x 2: weighted descaled event means, weighted spread */
    double *posteriors;           /* n_kmers: weights */
    uint8_t *observed;            /* n_kmers */
    /* HDP machine (hdpHmm_makeExpectationsHmm, continuousHmm.c:788-795): no emission expectations;
     * for each match transition whose posterior reaches the parameters' threshold, the path k-mer id
     * and the event's index in this read (cell_signal_updateExpectationsAndAssignments,
     * pairwiseAligner.c:795-817), this call's only, in the reference's order, up to
     * assignment_capacity (SA_E_OUTPUT beyond it; n_assignments is the count) */
    int64_t *assignment_kmers;
    int64_t *assignment_events;
    int64_t assignment_capacity;
    int64_t n_assignments;
} sa_expectations;

/* getExpectationsUsingAnchors with diagonalCalculation_Expectations (pairwiseAligner.c:1255-1275,
 * cell_signal_updateExpectations :763-793) on the plain FP64 form: the read's regions run in order in
 * one CTA; every transition posterior of the window's anti-diagonals is added in the reference's
 * order.  Canonical references only (SA_E_UNSUPPORTED for 'X'). */
sa_status sa_getExpectationsUsingAnchors(const sa_state_machine *sm, const char *reference, int64_t reference_length,
                                         const double *events, int64_t n_events, const int64_t *anchors,
                                         int64_t n_anchors, const sa_params *p, int32_t ragged_left,
                                         int32_t ragged_right, sa_expectations *ex);

/* Many reads' expectations in one launch (no signalAlign counterpart: signalMachine computes one
 * read's expectations per process, signalMachine.c:620-690, and the training script sums the
 * files).  One CTA walks read i's regions in order into ex[i], exactly as
 * sa_getExpectationsUsingAnchors does for one read (identical results); each read uses its own
 * scale / shift / var, ragged flags and machine.  read_status[i] is read i's status (ex[i] is
 * written only for SA_OK, and for SA_E_OUTPUT when its assignments overflowed); the call returns
 * SA_OK unless an argument, the parameters or a device step failed. */
sa_status sa_getExpectationsBatch(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_expectations *ex,
                                  int32_t *read_status);

/* The EM maximisation step (continuousPairHmm_normalize, continuousHmm.c:283-306): the transitions
 * divided by their row sums in place (hmmDiscrete_normalizeTransitions, discreteHmm.c:125-137); with
 * an event model (n_kmers rows of 5, the machine's match table when the expectations were made, as
 * continuousPairHmm_makeExpectationsHmm copies it, :201-212), each observed k-mer's level mean and
 * sd become sum(p * e) / sum(p) and sqrt(spread / sum(p)), a zero keeping the previous value.
 * event_model NULL: transitions only (the HDP machine's step). */
sa_status sa_normalizeExpectations(sa_expectations *ex, int64_t n_kmers, double *event_model);

/* continuousPairHmm_loadTransitionsIntoStateMachine (continuousHmm.c:321-339): the machine's nine
 * transitions become the logs of the normalised ones (gap-X -> gap-Y stays LOG_ZERO; gap-Y -> gap-X
 * becomes log(transitions[7])).  With an event model, continuousPairHmm_loadEmissionsIntoStateMachine
 * (:341-352) too (Gaussian machines only): match table level means and sds, gap-Y sds x 1.75, and
 * the gap-Y means at the index the reference writes them to (i + 5, not i * 5). */
sa_status sa_stateMachine_loadExpectations(sa_state_machine *sm, const double transitions[9],
                                           const double *event_model);

/* hmmContinuous_writeToFile (continuousHmm.c:872-884): continuousPairHmm_writeToFile (:354-406) for
 * the Gaussian machine, hdpHmm_writeToFile (:572-628) for the HDP machine (its assignments: the events'
 * means from `events`, rows of 4, and the k-mers), byte for byte; empty when a transition is NaN.
 * event_model NULL: the machine's match table.  The text is malloc'd (free with sa_free_text);
 * sa_writeExpectations writes it to `path` (opened with "w"). */
sa_status sa_formatExpectations(const sa_state_machine *sm, const sa_expectations *ex, const double *event_model,
                                const double *events, int64_t n_events, char **text, int64_t *length);
sa_status sa_writeExpectations(const char *path, const sa_state_machine *sm, const sa_expectations *ex,
                               const double *event_model, const double *events, int64_t n_events);

/* ---- before the path: anchor pairs from the guide alignment (signalMachine.c:615, :343-344) ---- */

/* one cigar operation of the guide alignment (AlignmentOperation of sonLib's PairwiseAlignment) */
typedef enum {
    SA_CIGAR_MATCH = 0,      /* PAIRWISE_MATCH: advances both sequences */
    SA_CIGAR_INDEL_X = 1,    /* PAIRWISE_INDEL_X: advances sequence 1 (the reference) only */
    SA_CIGAR_INDEL_Y = 2     /* PAIRWISE_INDEL_Y: advances sequence 2 (the read) only */
} sa_cigar_op_type;

typedef struct {
    int32_t op;              /* sa_cigar_op_type */
    int32_t pad;
    int64_t length;
} sa_cigar_op;

/* coordinates of a guide alignment (sonLib PairwiseAlignment: sequence 1 = reference, 2 = read) */
typedef struct {
    int64_t start1, end1;
    int32_t strand1;         /* 1 forward, 0 reverse (then start1 >= end1) */
    int32_t pad1;
    int64_t start2, end2;
    int32_t strand2;         /* must be 1 */
    int32_t pad2;
} sa_guide_alignment;

/* filterToRemoveOverlap (pairwiseAligner.c:1575-1616): from pairs sorted by (x, y), the ones that are
 * strictly increasing in both coordinates against every other pair kept.  out may alias pairs;
 * SA_E_ANCHORS if the input is not sorted. */
sa_status sa_filterToRemoveOverlap(const int64_t *pairs, int64_t n_pairs, int64_t *out, int64_t *n_out);

/* signalUtils_guideAlignmentToRebasedAnchorPairs (signalMachineUtils.c:142-164): rebases the
 * reference coordinates of *ga to 0 (flipping a reverse strand, as the reference does in place),
 * converts the cigar's match runs, less `trim` at both ends of each, into pairs
 * (convertPairwiseForwardStrandAlignmentToAnchorPairs, pairwiseAligner.c:1454-1478), sorts them and
 * filters overlaps.  out holds up to `capacity` pairs (SA_E_OUTPUT beyond, with *n_out the count
 * needed); SA_E_ARG if the cigar does not span the alignment's coordinates. */
sa_status sa_guideAlignmentToRebasedAnchorPairs(sa_guide_alignment *ga, const sa_cigar_op *ops, int64_t n_ops,
                                                int64_t trim, int64_t *out, int64_t capacity, int64_t *n_out);

/* signalUtils_getRemappedAnchorPairs (signalMachineUtils.c:166-170): (x, y) -> (x, event_map[y] -
 * event_map[map_offset]) (nanopore_remapAnchorPairsWithOffset, nanopore.c:438-450), then overlaps
 * filtered.  SA_E_ARG for an index outside event_map. */
sa_status sa_getRemappedAnchorPairs(const int64_t *anchors, int64_t n_anchors, const int64_t *event_map,
                                    int64_t map_length, int64_t map_offset, int64_t *out, int64_t *n_out);

/* ---- before the path: per-read scale / shift / drift / variance (signalMachineUtils.c:186-223) ---- */

/* NanoporeReadAdjustmentParameters (inc/nanopore.h:11-19) */
typedef struct {
    double scale, shift, var, shift_sd, scale_sd, var_sd, drift;
} sa_read_params;

/* one strand of a read for the estimation: its basecalled sequence, the event of each sequence
 * position (strand event map), and its event table (4 doubles per event: mean, noise, duration,
 * delta time) */
typedef struct {
    const sa_state_machine *sm;   /* the model: match table rows (mean, sd, noise mean, noise sd, lambda) */
    const char *read;
    int64_t read_length;
    const int64_t *event_map;     /* read_length entries */
    const double *events;
    int64_t n_events;
} sa_param_read;

/* nanopore_getOneDAssignmentsFromRead (nanopore.c:503-533): per k-mer of the read its event, the first
 * position of each event only; k-mer ids and (mean, noise, delta time) per assignment, up to
 * `capacity` (SA_E_OUTPUT beyond, *n_out the count); either output may be NULL */
sa_status sa_oneDAssignmentsFromRead(const sa_param_read *read, int64_t *kmer_ids, double *event_params,
                                     int64_t capacity, int64_t *n_out);

/* signalUtils_estimateNanoporeParams' fits for a batch of reads on the GPU, one CTA per read:
 * nanopore_compute_mean_scale_params with drift and variance (nanopore.c:650-781) and
 * nanopore_compute_noise_scale_params (:783-848) over the read's 1D assignments.  params[i] is
 * updated in place (scale, shift, drift, var, shift_sd, scale_sd, var_sd); read_status[i] is
 * SA_E_ARG for a read without assignments or with a singular system (the reference exits).  The
 * machine updates that follow in the reference are sa_stateMachine_setScaling and
 * sa_stateMachine_scaleNoise, and the drift correction sa_adjustEventsForDrift. */
sa_status sa_estimateNanoporeParams(const sa_param_read *reads, int64_t n_reads, sa_read_params *params,
                                    int32_t *read_status, void *stream);

/* nanopore_adjustEventsForDriftP (nanopore.c:535-540): mean -= delta time x drift, in place */
sa_status sa_adjustEventsForDrift(double *events, int64_t n_events, double drift);

/* ---- after the path: ordering, score and the posterior files (signalMachine.c:68-260, :715-728) ---- */

/* stList_sort(alignedPairs, sortByXPlusYCoordinate2) (pairwiseAligner.c:1434-1438): ascending x + y.
 * The reference sorts with qsort, which leaves the order of equal keys unspecified; this sort keeps
 * their input order. */
void sa_sortByXPlusYCoordinate(sa_aligned_pair *pairs, int64_t n_pairs);

/* scoreByPosteriorProbabilityIgnoringGaps (signalMachine.c:317-331): 100 x mean posterior */
double sa_scoreByPosteriorProbabilityIgnoringGaps(const sa_aligned_pair *pairs, int64_t n_pairs);

typedef enum {
    SA_OUTPUT_FULL = 0,             /* writePosteriorProbsFull */
    SA_OUTPUT_VARIANT_CALLER = 1,   /* writePosteriorProbsVC */
    SA_OUTPUT_ASSIGNMENTS = 2       /* writeAssignments */
} sa_output_format;

/* what outputAlignment needs besides the pairs and the model */
typedef struct {
    const char *read_label;
    const char *contig;
    const char *target;           /* the reference sequence the read was aligned to ('X' at degenerate sites) */
    int64_t target_length;
    int32_t strand;               /* 0 template, 1 complement */
    int32_t forward;              /* the guide alignment's strand */
    int64_t event_offset;         /* added to a pair's event index (the read's event map at the alignment start) */
    int64_t reference_offset;     /* the reference coordinate shift */
    const double *events;         /* the strand's whole event table, 4 doubles per event (mean, noise, duration, start) */
    int64_t n_events;
    double scale, shift, var, scale_sd;   /* NanoporeReadAdjustmentParameters */
} sa_output_read;

/* outputAlignment (signalMachine.c:240-260): the lines the reference appends to its posterior file,
 * byte for byte (printf formats of the reference), into a malloc'd NUL-terminated buffer (release with
 * sa_free_text).  Model means and noise come from sm's match table. */
sa_status sa_formatAlignment(sa_output_format fmt, const sa_state_machine *sm, const sa_output_read *rd,
                             const sa_aligned_pair *pairs, int64_t n_pairs, char **text, int64_t *length);
/* the same lines appended to the file at `path` */
sa_status sa_outputAlignment(sa_output_format fmt, const char *path, const sa_state_machine *sm,
                             const sa_output_read *rd, const sa_aligned_pair *pairs, int64_t n_pairs);
void sa_free_text(char *text);

/* ---- diagnostics ---- */
const char *sa_status_string(sa_status s);
/* number of kernel launches this process has made through the library (all entry points) */
int64_t sa_kernel_launch_count(void);
/* number of device and pinned-host allocations (cudaMalloc, cudaHostAlloc) the library has made in
 * this process (no counterpart in signalAlign: a diagnostic; memory pools reuse blocks, so a warm
 * steady state adds none) */
int64_t sa_allocation_count(void);
/* host time those allocation calls took, in milliseconds */
double sa_allocation_ms(void);
/* FP32 FMA issue rate of `device` in TFLOP/s, measured by a short probe kernel (the denominator of
 * the engine's compute roofline; no counterpart in signalAlign) */
sa_status sa_measure_fp32_peak(int32_t device, double *tflops);

#ifdef __cplusplus
}
#endif

#endif /* SA_B200_H_ */
