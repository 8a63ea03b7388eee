// Internal declarations shared by the host planner (sa_host.cpp) and the CUDA kernels
// (sa_fp64.cu, sa_fp32.cu).  Nothing here is part of the C ABI.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "sa_b200.h"

namespace sa {

constexpr int kEventParams = 4;                 // NB_EVENT_PARAMS (inc/nanopore.h:4)
constexpr double kPairProb1 = 10000000.0;       // PAIR_ALIGNMENT_PROB_1 (inc/pairwiseAligner.h:27)
constexpr double kLogPointOne = -2.3025850929940455;  // gap-X emission, stateMachine.c:1282, :1472-1474
constexpr int kMaxK = 12;

// ----------------------------------------------------------------------------------------------
// state machine: host copy of the reference tables, device copies for both kernel forms
// ----------------------------------------------------------------------------------------------
struct HdpTables {
    bool present = false;
    double grid_start = 0, grid_stop = 0;
    int64_t grid_length = 0;
    int64_t n_rows = 0;
    std::vector<double> grid;       // linspace (hdp_math_utils.c:497-509)
    std::vector<double> density;    // n_rows x grid_length
    std::vector<double> slope;      // n_rows x grid_length
    std::vector<int64_t> kmer_row;  // n_kmers
    std::vector<char> kmer_observed;  // n_kmers: the k-mer's own DP is observed (hdp_check_for_observed)
};

// FP32 per-k-mer emission constants (one 32-byte record per k-mer), derived on the host in FP64
// from the reference tables:
//   mu, 1/sd_match, 1/sd_gapy, k_m = -log(2 pi) - log(sd_match) + 0.5 log(lambda),
//   k_y = -log(2 pi) - log(sd_gapy) + 0.5 log(lambda), 1/noise_mean, lambda/2, gap-X log probability
struct __align__(16) KmerConst32 {
    float mu, inv_sd_m, inv_sd_y, k_m;
    float k_y, inv_nu, half_lambda, gapx;
};

struct DeviceModel {
    int device = 0;
    // FP64 tables (reference layout)
    double *match = nullptr, *gapy = nullptr, *gapx = nullptr;
    double *klog = nullptr;   // per k-mer: log sd (match, gap-Y), log lambda (match, gap-Y)
    double *hdp_grid = nullptr, *hdp_density = nullptr, *hdp_slope = nullptr;
    int64_t *hdp_kmer_row = nullptr;
    // FP32 tables
    KmerConst32 *kc32 = nullptr;
    float *gapx32 = nullptr;
};

}  // namespace sa

struct sa_state_machine {
    sa_machine_type type;
    sa_emission emission;
    std::string alphabet;            // sorted (sequence_prepareAlphabet, pairwiseAligner.c:294-323)
    int32_t kmer_length = 0;
    int64_t n_kmers = 0;
    double t[SA_N_TRANSITIONS];
    double scale = 1.0, shift = 0.0, var = 1.0;
    std::vector<double> match, gapy, gapx;
    sa::HdpTables hdp;
    std::vector<std::string> kmer_strings;   // interned path k-mers, built on first use
    sa::DeviceModel dev;
    bool dev_dirty = true;
};

namespace sa {

// ----------------------------------------------------------------------------------------------
// host planning
// ----------------------------------------------------------------------------------------------
struct Window {
    int32_t T;      // traced back to (exclusive lower end of the posterior range)
    int32_t D;      // traceback diagonal (backward end point)
    int32_t from;   // last diagonal whose posteriors this window emits
    int32_t at_end;
};

struct Region {
    int64_t x1 = 0, y1 = 0;          // offset of the region in read coordinates
    int64_t lX = 0, lY = 0;          // k-mers, events
    int32_t ragged_left = 0, ragged_right = 0;
    std::vector<int32_t> xmy_l, xmy_r;   // per anti-diagonal 0..lX+lY
    std::vector<Window> windows;
    int64_t cells = 0;
    int32_t max_width = 0;
};

// band_construct (pairwiseAligner.c:131-182); returns SA_E_ANCHORS on bad anchors
sa_status band_construct(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t expansion,
                         int64_t *xmy_l, int64_t *xmy_r);

// getSplitPoints (pairwiseAligner.c:1730-1757)
sa_status split_points(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, int64_t limit,
                       bool ragged_left, bool ragged_right, std::vector<int64_t> &regions);

// getPosteriorProbsWithBandingSplittingAlignmentsByLargeGaps (pairwiseAligner.c:1773-1837) minus the DP:
// region geometry, band, traceback windows (getPosteriorProbsWithBanding :1319-1333, :1350)
sa_status plan_regions(const int64_t *anchors, int64_t n_anchors, int64_t lX, int64_t lY, const sa_params &p,
                       bool ragged_left, bool ragged_right, std::vector<Region> &regions);

sa_status check_params(const sa_params &p);

// path k-mers of one reference: per column x (1..lX) the ids of its paths (single id when no 'X')
struct PathTable {
    int64_t lX = 0;
    bool multi = false;              // some column has more than one path
    std::vector<int32_t> first;      // lX + 1 entries; column x's paths are ids[first[x] .. first[x+1])
    std::vector<int32_t> ids;        // k-mer ids; column 0 holds the NULL path (-1)
};

const char *degenerate_options(int32_t degenerate);
sa_status build_paths(const sa_state_machine *sm, const char *reference, int64_t lX, int32_t degenerate,
                      PathTable &pt);

// device model upload (both kernel forms)
sa_status ensure_device_model(sa_state_machine *sm);

// the plain FP64 form's per-k-mer logs (DeviceModel::klog) from the resident tables, on the device
sa_status compute_kmer_logs(sa_state_machine *sm);

// The batched FP32 form takes the extra-event (gap-Y) emission's level mean, noise mean and noise
// lambda from the match table and only the level sd from the gap-Y table.  True when the machine's
// tables agree on those three fields for every k-mer (tables read from a .model file, and scaled by
// scaleModel / scaleNoise, always do); reads of other machines run in the plain FP64 form.
bool gapy_follows_match(const sa_state_machine *sm);
void free_device_model(sa_state_machine *sm);

void count_launch(int64_t n = 1);

// every cudaMalloc / cudaHostAlloc of the library goes through these two, which count the
// successful ones (sa_allocation_count)
cudaError_t device_malloc(void **ptr, size_t bytes);
cudaError_t pinned_malloc(void **ptr, size_t bytes);

// the machine's device tables are current (no change since its last upload), read under the lock
// that guards the upload
bool model_resident(const sa_state_machine *sm);

// memory blocks reused across batches (sa_memory.cpp): device and pinned host blocks go back to a
// free list; heap blocks (for callers that must not touch the CUDA allocators) are freed
enum class MemKind { Device, Pinned, Heap };
struct MemBlock {
    void *ptr = nullptr;
    size_t bytes = 0;
    int device = -1;
    MemKind kind = MemKind::Heap;
};
sa_status mem_get(MemKind kind, int device, size_t bytes, MemBlock &out);
void mem_put(MemBlock &b);

// forward-segment planning shared by both forms (sa_fp32.cu): the policy (cap, -1 off, 0 automatic;
// warm-up), the automatic cap's floor, a region's warm-up and its cuts (window indices)
void segment_policy(int32_t &target, int32_t &warm);
int64_t segment_min();
int32_t segment_warm(const Region &rg, int32_t warm);
void segment_cuts(const Region &rg, int64_t target, int32_t warm, std::vector<int32_t> &cuts);

// batches bound to one caller-provided device area instead of their own allocations (sa_fp32.cu)
sa_status batch_plan_host(const sa_read *reads, int64_t n_reads, const sa_params *p, sa_batch **out);
int batch_device(const sa_batch *b);
bool batch_models_resident(const sa_batch *b);
// bytes of the area that holds every device buffer of `b`; with base != nullptr the batch's device
// pointers are set into [base, base + bytes), each buffer 256-byte aligned
size_t batch_bind_scratch(sa_batch *b, unsigned char *base);
// frees the host side only (the device area belongs to the caller)
void batch_release_host(sa_batch *b);

// Per-read completion of a batch (the serving loop): the worker kernel's group that finishes a
// read's last traceback window gathers the read's pairs into the packed output and writes the
// read's record to mapped host memory, `done` last after a system-scope fence.  Reads that run no
// window in the FP32 kernels (plan errors, plain-form reads, reads without windows) and reads of a
// run whose bounded wait gave up get no record; their results come from sa_batch_download.  A
// record belongs to the batch's latest run when its `done` equals batch_run_seq (runs are numbered
// from 1, so records need no clearing between runs).
struct ReadDone {
    int64_t first_pair;       // in the packed output
    int64_t n_pairs;
    double log_likelihood;    // the read's regions' totals summed in region order
    int32_t status;           // the read's device status (SA_OK or SA_E_OUTPUT)
    int32_t done;             // the publishing run's number
};
// before sa_batch_run (batches that own their device memory): every later run publishes its reads;
// the gather launch after the worker is then left out
sa_status batch_publish_reads(sa_batch *b);
// n_reads records (nullptr before batch_publish_reads) and the number of the latest run
const ReadDone *batch_read_records(const sa_batch *b);
int32_t batch_run_seq(const sa_batch *b);
// copies a published read's pairs into dst on `stream` and waits for the copy
sa_status batch_fetch_read(const sa_batch *b, const ReadDone &rec, sa_aligned_pair *dst, cudaStream_t stream);
// timing events of the last run: before the emission kernel, after the worker kernel
bool batch_run_events(const sa_batch *b, cudaEvent_t *start, cudaEvent_t *end);

// the plain FP64 form over a set of reads (sa_fp64.cu): every region one CTA of one launch, F and
// B in rings of the longest traceback window.  Used by the single-read entry and, inside batches,
// for reads whose references have degenerate ('X') positions.
struct PlainSet;
// segments: cut long regions into forward segments (alignment runs; not the expectations mode)
sa_status plain_create(const sa_read *reads, int64_t n_reads, const sa_params &p, size_t max_bytes, PlainSet **out,
                       bool segments = false);
// scale of the set's stitch tolerance (negative: every stitch disagrees and its region re-runs whole)
void plain_set_stitch_tolerance(PlainSet *s, double scale);
// forward segments of the plain form in use: stitches and regions re-run whole at the last download
void plain_segment_info(const PlainSet *s, int64_t *n_tasks, int64_t *n_stitches, int64_t *n_redone);
sa_status plain_upload(PlainSet *s, cudaStream_t stream);
sa_status plain_run(PlainSet *s, cudaStream_t stream);
sa_status plain_download(PlainSet *s, cudaStream_t stream);
int plain_device(const PlainSet *s);
int64_t plain_cells(const PlainSet *s);
size_t plain_in_bytes(const PlainSet *s);
sa_status plain_read_status(const PlainSet *s, int64_t r);
const std::vector<sa_aligned_pair> &plain_pairs(const PlainSet *s, int64_t r);
double plain_log_likelihood(const PlainSet *s, int64_t r);
void plain_destroy(PlainSet *s);

#define SA_CUDA_TRY(expr)                                   \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return SA_E_CUDA;            \
    } while (0)

}  // namespace sa
