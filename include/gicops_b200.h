/* gicops_b200: B200-native peptide-search query path (DSLIM fragment-ion index
 * lookup -> BYC shared-peak scorecard -> hyperscore -> top-K -> score histogram ->
 * tail-fit e-value) behind a plain C ABI.
 *
 * The entry points replace the reference's query-path boundary (paths are
 * relative to the reference project, mhaseeb123/gicops):
 *   hcp::gpu::cuda::s3::initialize / search / deinitialize / getBYC / getScorecard /
 *   reset_dScores   source/core/include/cuda/superstep3/kernel.hpp:88-100
 *   hcp::gpu::cuda::s1::getdIndex (index residency)   source/core/cuda/superstep1/kernel.cu:310-358
 *   hcp::gpu::cuda::s4::processResults (tail fit + results) source/core/cuda/superstep4/kernel.cu:491-596
 *   DSLIM_QuerySpectrum (CPU query path)           source/core/include/dslim.h:196
 *   DSLIM_Construct + LBE_* (host index build)     source/core/dslim.cpp:46-153, source/core/lbe_internal.cpp
 *
 * Conventions: every call returns a gx_status (codes mirror source/core/include/slmerr.h)
 * and never exits the process; gx_last_error() gives the message of the calling
 * thread's last failure.  Calls are thread-compatible: use one gx_workspace per host
 * thread.  Device-pointer calls are stream-ordered and do not synchronise.
 */
#ifndef GICOPS_B200_H
#define GICOPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (source/core/include/slmerr.h:24-43) ------------------------------ */
typedef int32_t gx_status;
#define GX_SUCCESS             0
#define GX_ERR_INVLD_MEMORY    (-3001)
#define GX_ERR_INVLD_PARAM     (-3002)
#define GX_ERR_INVLD_INDEX     (-3003)
#define GX_ERR_INVLD_SIZE      (-3004)
#define GX_ERR_FILE_NOT_FOUND  (-3006)
#define GX_ERR_BAD_MEM_ALLOC   (-3007)
#define GX_ERR_INVLD_PTR       (-3008)
#define GX_ERR_INVLD_MOD       (-3010)
#define GX_ERR_NOT_ENOUGH_DATA (-3012)
/* additions (no counterpart in slmerr.h): CUDA failure, device-side guard tripped */
#define GX_ERR_CUDA            (-3050)
#define GX_ERR_DEVICE_GUARD    (-3051)

#define GX_HIST_BINS 802      /* 2 + MAX_HYPERSCORE*10 (source/core/include/expeRT.h:115) */
#define GX_MAX_HEAP  31       /* largest top-K heap capacity supported (topmatches <= 31) */
#define GX_MAX_LENGTHS 64     /* peptide lengths per index */
#define GX_MAX_PEAKS 1024     /* peaks per spectrum (the reference's QALEN is 100) */

/* ---- index (source/core/include/slm_dsts.h:146-346) --------------------------------- */

/* One index entry (pepEntry, slm_dsts.h:146): precursor mass, sequence id within its
 * length, modification site mask, modification numbers (4 bits per modified site). */
typedef struct {
    float mass;
    uint32_t seqid;
    uint64_t sites;
    uint32_t modnum;
    uint32_t pad;
} gx_pep_entry;

/* Query-path view of one per-length index (Index + its single ionIndex chunk). */
typedef struct {
    uint32_t peplen;      /* L */
    uint32_t npep;        /* N entries (peptides + variants), ascending mass */
    uint32_t speclen;     /* ions per entry = 2*(L-1)*maxz */
    uint32_t pad;
    const float *mass;    /* [N] entry masses, ascending */
    const uint32_t *bA;   /* [nbins] CSR offsets per 0.01 Da fragment bin (DSLIM_Matrix.bA) */
    const uint32_t *iA;   /* [N*speclen] ion ids pepid*speclen+pos, ascending in a bin (DSLIM_Matrix.iA) */
} gx_length_desc;

typedef struct gx_index gx_index;          /* device-resident index (opaque) */
typedef struct gx_workspace gx_workspace;  /* device scratch for one host thread (opaque) */

/* Upload (copy) the per-length host arrays into HBM on `device`; replaces
 * s1::getdIndex.  nbins must be max_mass*scale + 1.  Lengths must be given in the
 * order their results are to be reported (idxoffset = position in this array). */
gx_status gx_index_upload(const gx_length_desc *lens, int32_t nlen, uint32_t nbins, int32_t device,
                          gx_index **out);
gx_status gx_index_free(gx_index *ix);
/* bytes held in HBM by an index */
uint64_t gx_index_bytes(const gx_index *ix);
/* Write a device index to a file, every array as the device holds it, and load such a file
 * onto a device without building anything (the large configuration's 27 GB index takes 20 s
 * to build from host arrays).  The file records the library's entry-block size and layout
 * version; a file of another layout, a truncated file or one of another kind is refused
 * (GX_ERR_INVLD_INDEX, GX_ERR_NOT_ENOUGH_DATA).  Copies go through a 64 MB pinned buffer.
 * No counterpart in the reference, which rebuilds its index in every run and caches only
 * preprocessed spectra (source/core/msquery.cpp:542-721). */
gx_status gx_index_save(const gx_index *ix, const char *path);
gx_status gx_index_load(const char *path, int32_t device, gx_index **out);

/* ---- host index builder (LBE_CountPeps/Initialize + MODS_GenerateMods + DSLIM_Construct) */
typedef struct {
    char residues[4];     /* residues the modification applies to, NUL padded */
    double mass;          /* Da; stored as (uint)(mass*scale) like argp.hpp:359 */
    uint32_t max_per_pep; /* per-peptide limit for this modification */
} gx_mod;

typedef struct {
    uint32_t maxz;        /* fragment charges indexed */
    uint32_t scale;       /* bins per Da (100) */
    uint32_t min_mass, max_mass;   /* precursor mass filter (500, 5000) */
    uint32_t nmods;       /* number of gx_mod entries */
    uint32_t mods_per_pep;/* total modified residues per peptide (0: no variants) */
    const gx_mod *mods;
    int32_t threads;      /* host threads (<=0: all) */
} gx_build_params;

typedef struct gx_host_length gx_host_length;  /* host-side per-length index (opaque) */

/* Build the index of one peptide length from `npep` sequences of length L
 * (row-major, no separators, the order of the L.peps file). */
gx_status gx_build_length(const char *seqs, uint32_t npep, uint32_t L, const gx_build_params *bp,
                          gx_host_length **out);
/* Accessors: the descriptor points into the object; entries, kept sequences
 * (peptides that passed the mass filter, index seqid order). */
gx_status gx_host_length_desc(const gx_host_length *h, gx_length_desc *desc);
const gx_pep_entry *gx_host_length_entries(const gx_host_length *h);
const char *gx_host_length_seqs(const gx_host_length *h, uint32_t *npep_kept);
void gx_host_length_free(gx_host_length *h);
/* Entries of one length only (mass filter, variant enumeration, mass sort: the steps
 * of gx_build_length before the fragment ions), for gx_index_build, which computes the
 * ions on the GPU.  The descriptor of such a length has bA = iA = NULL. */
gx_status gx_build_length_entries(const char *seqs, uint32_t npep, uint32_t L, const gx_build_params *bp,
                                  gx_host_length **out);

/* ---- device index builder (DSLIM_Construct's ion and CSR stage, dslim.cpp:231-504 with
 * the ion arithmetic of utils.cpp:161-474, on the GPU, plus s1::getdIndex) ------------
 * Builds the device-resident index on `device` from host lengths (gx_build_length or
 * gx_build_length_entries with the same gx_build_params, in idxoffset order): fragment
 * ions, bA / iA and the block layout are computed on the GPU and equal those of
 * gx_index_upload of the host-built lengths.  At most 2^31 - 1 ion ids per length. */
gx_status gx_index_build(gx_host_length *const *lens, int32_t nlen, const gx_build_params *bp, int32_t device,
                         gx_index **out);
/* Copy one length of a device index to the host (any pointer may be NULL): bA [nbins],
 * iA [npep*speclen] with ids as the device holds them (2*entry + (y ion)), iAb
 * [npep*speclen] (block-local 16-bit ids), mass [npep].  No counterpart in the reference. */
gx_status gx_index_read_length(const gx_index *ix, int32_t i, uint32_t *bA, uint32_t *iA, uint16_t *iAb,
                               float *mass);

/* ---- query preprocessing (MSQuery::convertAndprepMS2bin, msquery.cpp:137-336) -------- */
typedef struct gx_ms2_file gx_ms2_file;   /* raw spectra read from an MS2 file (opaque) */

/* Raw spectra as the reference collects them before peak picking.  Spectrum s owns the
 * values [seg[s], seg[s+1]) (normally size[s] of them; values before a file's first S
 * line belong to the first spectrum, whose size counts only the lines after its S). */
typedef struct {
    uint32_t nspec, nvalues;
    const uint32_t *seg;     /* [nspec + 1] */
    const uint32_t *size;    /* [nspec] */
    const int32_t *mz;       /* [nvalues] (int)(m/z * scale) */
    const int32_t *intn;     /* [nvalues] (int)(intensity * 100) */
    const float *prec;       /* [nspec] precursor M+H from the Z line */
    const int32_t *charge;   /* [nspec] */
    const float *rtime;      /* [nspec] */
} gx_ms2_raw;

/* Read an MS2 text file with the reference's parsing rules (the first half of
 * convertAndprepMS2bin); scale = bins per Da (100). */
gx_status gx_ms2_read(const char *path, uint32_t scale, gx_ms2_file **out);
gx_status gx_ms2_desc(const gx_ms2_file *f, gx_ms2_raw *raw);
void gx_ms2_free(gx_ms2_file *f);

/* Peak picking and intensity normalisation on the GPU (MSQuery::pickpeaks,
 * msquery.cpp:338-423, with the key-value quicksort of include/keyval.h:49-129): per
 * spectrum the first size[s] values of its segment are sorted by intensity (the
 * reference's exact quicksort, so ties keep its order), the top one is set to base_int
 * and the others scaled by base_int / top (truncated to int), and the peaks from the
 * top down to the first one below min_int, at most qalen, are kept: the last `kept`
 * values of the segment, in ascending intensity.  Device arrays, stream-ordered;
 * mz_dev / intn_dev are sorted and scaled in place; out_idx_dev [nspec + 1] receives the
 * kept peaks' CSR offsets and out_mz_dev / out_intn_dev (capacity nvalues) the peaks.
 * The reference's defaults: base_int 100000, min_int 1000, qalen 100. */
gx_status gx_pickpeaks_device(uint32_t nspec, const uint32_t *seg_dev, const uint32_t *size_dev, int32_t *mz_dev,
                              int32_t *intn_dev, int32_t base_int, int32_t min_int, uint32_t qalen,
                              uint32_t *out_idx_dev, int32_t *out_mz_dev, int32_t *out_intn_dev, void *stream);

/* ---- search ------------------------------------------------------------------------ */
typedef struct {
    double dM;            /* precursor tolerance (Da), used when gx_queries.dM is NULL */
    uint32_t dF;          /* fragment tolerance (bins) */
    uint32_t scale;       /* bins per Da */
    double max_mass;      /* Da */
    uint32_t min_shp;     /* shared peaks for a candidate PSM (4) */
    uint32_t min_cpsm;    /* candidate PSMs for an e-value (4); 0 acts as 1 (an e-value needs a
                           * top PSM; the reference reads its empty heap there) */
    uint32_t topmatches;  /* heap capacity = 2^floor(log2(t)+0.999) - 1 (dslim.cpp:438-444) */
    uint32_t flags;       /* GX_FLAG_* */
    double expect_max;    /* PSMs with e >= expect_max are not reported */
} gx_params;

#define GX_FLAG_WIDE_SCORECARD 1u   /* force the 12-byte scorecard (testing) */
#define GX_FLAG_PLAIN          2u   /* one spectrum per CTA, no work queue (plain path) */

/* Spectra in the reference's Queries<int> layout (slm_dsts.h:520-658). */
typedef struct {
    uint32_t nspec;
    uint32_t npeaks;      /* idx[nspec] */
    const uint32_t *idx;  /* [nspec+1] */
    const int32_t *moz;   /* [npeaks] m/z bins */
    const int32_t *intn;  /* [npeaks] intensities */
    const float *prec;    /* [nspec] precursor masses */
    const int32_t *charge;/* [nspec] or NULL (reported; a feature of the learned tail) */
    const double *dM;     /* [nspec] per-spectrum tolerance (Da) or NULL */
} gx_queries;

/* One candidate PSM (hCell's query-path fields, slm_dsts.h:661-761). */
typedef struct {
    float hyperscore;
    int32_t psid;         /* entry index within its length */
    uint16_t idxoffset;   /* length index */
    uint16_t sharedions;
    uint16_t totalions;
    uint16_t pad;
} gx_cell;

/* Per-spectrum result.  status bits: 1 = cpsms >= max(min_cpsm, 1) (e-value computed),
 * 2 = e_x < expect_max (a PSM the reference prints), 4 = a shared-ion count above
 * MAX_SHDPEAKS (80) was clamped, 8 = the 12-byte scorecard was used, 16 = the e-value
 * comes from the learned tail (gx_tail_apply), 32 = GX_STATUS_PEAK_LIMIT: the spectrum has
 * more than GX_MAX_PEAKS peaks and was not searched (every other field zero, its histogram
 * and heap rows empty; gx_search_host also returns GX_ERR_DEVICE_GUARD for the batch). */
#define GX_STATUS_PEAK_LIMIT 32
typedef struct {
    int32_t cpsms;
    int32_t status;
    gx_cell top;          /* minHeap::getMax() of the reference's top-K heap */
    int32_t maxhyp;       /* (int)(top.hyperscore*10+0.5) */
    int32_t mu, beta;     /* tail-fit slope/intercept x1e6 truncated (Results.mu/beta) */
    int32_t stt1, end1;   /* tail-fit curve region */
    int32_t pad;
    double slope, icpt;   /* unquantized FP64 fit */
    double e_x;           /* e-value as the reference computes it */
    double e_fp64;        /* e-value from the unquantized fit */
} gx_result;

/* ---- index-sharded search: merge of the ranks' partial results ----------------------
 * Replaces the reference's exchange of partial results between MPI ranks that own
 * peptide subsets (source/core/dslim_score.cpp:199-388, through files).  Every rank
 * searched all nspec spectra against its own lengths (gx_search_device with heap and
 * histogram outputs); after the histograms and candidate counts are summed over ranks
 * and the ranks' cells and statuses gathered (NCCL), this writes the global top cells
 * [nspec][cap] (cap = gx_heap_capacity(p->topmatches); top_dev may be NULL) ordered by
 * hyperscore descending, then global length index and entry ascending, and the result
 * records with the tail fit of the summed histogram.  cells_dev [world][nspec][k] with
 * rank-local idxoffset, status_dev [world][nspec], lut_dev [world][GX_MAX_LENGTHS] =
 * global length index of each rank-local one, hist_dev [nspec][GX_HIST_BINS] and
 * cpsms_dev [nspec] summed.  Stream-ordered. */
gx_status gx_merge_shards_device(uint32_t nspec, int32_t world, uint32_t k, const gx_cell *cells_dev,
                                 const int32_t *status_dev, const uint16_t *lut_dev, const uint32_t *hist_dev,
                                 const int32_t *cpsms_dev, const gx_params *p, gx_cell *top_dev, gx_result *out_dev,
                                 void *stream);

/* Workspace sized for up to max_spec spectra / max_peaks peaks per call. */
gx_status gx_workspace_create(const gx_index *ix, uint32_t max_spec, uint32_t max_peaks, gx_workspace **out);
gx_status gx_workspace_free(gx_workspace *ws);

/* ---- launch shape of the batched path and its autotuner (no counterpart in the
 * reference, whose launch shape is fixed: superstep3/kernel.cu:588-598) ---------------
 * chunks_per_lane: 16-byte id chunks (8 ids) each lane loads per work unit (the bucket
 * chunk), 1..3; ctas_per_sm: persistent CTAs per SM, each on its own spectrum, 1..2;
 * tile: candidates per shared-memory scorecard tile (the scorecard partition width), a
 * multiple of 32 from 1024 to the index's block of 11,264 entries; sorted: 1 takes the
 * spectra heaviest first (a sort by scan volume), 0 in batch order; pipeline: 1 runs the
 * spectra with the 8-byte scorecard and at most 256 bin intervals through the pipelined
 * kernel (one CTA of 32 warps per SM, one tile scored while the next streams into a second
 * scorecard; ctas_per_sm then applies to the others).  Results do not depend on the shape.
 * A new workspace starts at {2, 2, 11264, 1, 0}. */
typedef struct {
    uint32_t chunks_per_lane;
    uint32_t ctas_per_sm;
    uint32_t tile;
    uint32_t sorted;
    uint32_t pipeline;            /* 1: one CTA of 32 warps per SM with two scorecard tiles, scoring one
                                   * tile while streaming the next (tile = the whole block only) */
} gx_tiles;
/* CUDA graphs for the batched path's launch sequence (on = 1; 0 releases them).  The
 * sequence (k_prep, sort, k_search_batched, k_tailfit, learned tail) is captured on the
 * workspace's stream the first time a combination of query and output buffers, parameters,
 * launch shape and attached tail is seen, and replayed afterwards (the last 4 kept); it is
 * ordered after the caller's earlier work on its stream, and before its later work, by
 * events.  The plain path and calls made while gx_profile_enable is on launch directly.
 * No counterpart in the reference (one launch per kernel per batch). */
gx_status gx_workspace_set_graph(gx_workspace *ws, int32_t on);
gx_status gx_workspace_get_tiles(const gx_workspace *ws, gx_tiles *t);
gx_status gx_workspace_set_tiles(gx_workspace *ws, const gx_tiles *t);
#define GX_TUNE_MAX 32
typedef struct {
    gx_tiles best;
    uint32_t ncand;               /* candidates timed (0 when taken from the cache) */
    uint32_t cached;              /* 1: an earlier call's choice for the same workload shape */
    gx_tiles cand[GX_TUNE_MAX];
    float ms[GX_TUNE_MAX];        /* median of `reps` timed searches of the sample, per candidate */
} gx_tune_result;
/* Times every candidate shape (chunks 1-3 x CTAs per SM 1-2 x tile {block, 3/4 block} x
 * sorted or not, and the pipelined kernel with chunks 1-3, sorted or not) on the sample q_dev (device buffers: a few thousand spectra of the
 * workload), one warm-up and `reps` timed searches each on `stream`, sets the fastest on
 * the workspace and caches it for the workload shape (index, tolerance or per-spectrum
 * tolerances, dF, min_shp, heap capacity, flags, maxz).  With use_cache, a cached choice
 * for the same shape is set without timing anything.  Synchronises the stream; writes
 * the workspace's own result buffer only. */
gx_status gx_autotune(gx_index *ix, gx_workspace *ws, const gx_queries *q_dev, const gx_params *p, uint32_t reps,
                      uint32_t use_cache, gx_tune_result *out, void *stream);

/* Search with HOST buffers (the drop-in for s3::search + s4::processResults):
 * copies queries in, runs the path, copies results out, synchronises.
 * heap_out (optional): [nspec * cap] final heap arrays; hist_out (optional):
 * [nspec * GX_HIST_BINS] score histograms. */
gx_status gx_search_host(gx_index *ix, gx_workspace *ws, const gx_queries *q, const gx_params *p,
                         gx_result *out, gx_cell *heap_out, uint32_t *hist_out);

/* Search with DEVICE buffers already resident in HBM (stream-ordered, no sync). */
gx_status gx_search_device(gx_index *ix, gx_workspace *ws, const gx_queries *q_dev, const gx_params *p,
                           gx_result *out_dev, gx_cell *heap_dev, uint32_t *hist_dev, void *stream);

/* Search with DEVICE buffers and no device allocation of any kind (no counterpart in
 * the reference).  For callers that cannot call cudaMalloc: hosts whose memory pool owns
 * every byte of the device, callers with a memory budget fixed at start-up, or code where
 * an allocation could block or fail at an unsafe point.  It runs the plain path
 * (GX_FLAG_PLAIN semantics) with its scratch in a fixed file-scope device array of
 * GX_NOALLOC_MAX_WINDOWS windows (4 MiB, held by every device that loads the library until
 * exit); batches with nspec * nlen above that are rejected with GX_ERR_INVLD_SIZE.  The
 * first call on a device looks the array up and sets the kernel up on that device: make
 * it before any stream capture.  All calls share the array; calls that overlap on the GPU
 * race and must be serialised by the caller.  Stream-ordered, no synchronisation: a
 * spectrum over GX_MAX_PEAKS peaks is reported through its status (GX_STATUS_PEAK_LIMIT).
 * A cudaDeviceReset (or release of the primary context) drops the array's contents; the
 * next call on that device notices the new context and sets the array up again. */
#define GX_NOALLOC_MAX_WINDOWS (1u << 19)
gx_status gx_search_device_noalloc(gx_index *ix, const gx_queries *q_dev, const gx_params *p, gx_result *out_dev,
                                   gx_cell *heap_dev, uint32_t *hist_dev, void *stream);

/* ---- streamed search of a batch in host memory --------------------------------------
 * Replaces the reference's batch feed to its GPU path: a ring of host query buffers
 * (source/core/dslim_query.cpp:183-203), each batch uploaded synchronously before its
 * search (dQueries::H2D, source/core/cuda/superstep3/kernel.cu:192-206).  A streamer owns
 * a workspace for `chunk` spectra and two sets of device query and result buffers: a host
 * batch of any size is searched chunk by chunk, the upload of one chunk (one
 * cudaMemcpyAsync per array, on an upload stream) and the download of another's results
 * (a download stream) overlapping the search of a third (the workspace's stream).  The
 * results equal one gx_search_device call over the whole batch.  Host arrays should be
 * pinned (cudaHostAlloc / cudaHostRegister) for the copies to overlap; pageable memory
 * gives the same results with the copies serialised.  max_peaks = peaks per chunk the
 * buffers hold (0: chunk * 160).  A learned tail is attached through
 * gx_workspace_set_tail(gx_streamer_workspace(s), ...). */
typedef struct gx_streamer gx_streamer;
typedef struct {
    uint32_t chunks;
    uint32_t pad;
    double total_ms;      /* first upload to last download, GPU clock */
    double upload_ms;     /* summed over chunks: host-to-device copies */
    double search_ms;     /* summed over chunks: the search launch sequence */
    double download_ms;   /* summed over chunks: device-to-host copies of the results */
} gx_stream_stats;
gx_status gx_streamer_create(gx_index *ix, uint32_t chunk, uint32_t max_peaks, gx_streamer **out);
gx_status gx_streamer_free(gx_streamer *s);
gx_workspace *gx_streamer_workspace(gx_streamer *s);
/* Search q (HOST arrays, idx[0] = 0) into out (HOST, q->nspec records); stats may be NULL
 * (when given, each chunk's copies and search are timed with events, which adds a little
 * host overhead).  Synchronises before returning; GX_ERR_DEVICE_GUARD if a spectrum had
 * more than GX_MAX_PEAKS peaks (its record carries GX_STATUS_PEAK_LIMIT), GX_ERR_INVLD_SIZE
 * before any work if a chunk holds more peaks than the streamer's buffers. */
gx_status gx_search_stream(gx_streamer *s, const gx_queries *q, const gx_params *p, gx_result *out,
                           gx_stream_stats *stats);

/* Algorithmic traffic of the path, per spectrum (host arrays, for roofline figures):
 * ids_out[s] = ion ids inside the precursor window of every distinct probed bin,
 * bins_out[s] = distinct probed bins, both summed over lengths with a non-empty
 * window.  No counterpart in the reference (measurement only). */
gx_status gx_traffic_host(const gx_length_desc *lens, int32_t nlen, const gx_queries *q, const gx_params *p,
                          int64_t *ids_out, int64_t *bins_out, int32_t threads);

/* Heap capacity the reference uses for `topmatches` (dslim.cpp:438-444). */
int32_t gx_heap_capacity(uint32_t topmatches);

/* Hyperscore table: out[i] = sum_{k<=i} log10(k), i = 0..80 (utils.h:115-131). */
void gx_lgfact(double *out81);

/* Kernel timing: when enabled, every kernel the library launches is bracketed by
 * CUDA events recorded on its own stream.  gx_profile_read synchronises those
 * events and returns per-kernel totals (launches, milliseconds); enabling again
 * clears them.  No counterpart in the reference (it times with host clocks). */
typedef struct {
    char name[40];
    uint64_t launches;
    double total_ms;
} gx_kernel_time;
gx_status gx_profile_enable(int32_t on);
int32_t gx_profile_read(gx_kernel_time *out, int32_t cap);

/* ---- learned tail (no counterpart in the reference) ---------------------------------
 * A small MLP that predicts a query's expeRT log-survival line from its score histogram,
 * for queries whose histogram holds too few candidates for a stable plain fit
 * (source/core/expeRT.cpp ModelTailFit is the plain fit it stands in for).
 *
 * Input (GX_TAIL_IN features, bf16): log10(1 + count) of the GX_TAIL_WINDOW histogram
 * bins from the first non-empty bin b0, then log10(candidates), precursor mass / 1000,
 * charge, (maxhyp - b0) / 100.  Network 132 -> 256 -> 256 -> 2 with GELU (erf form);
 * bf16 weights and activations, fp32 accumulation on the tensor cores, fp32 master
 * weights and Adam.  Output: the line's slope (per histogram bin) and its value at
 * maxhyp (log10 survival fraction); the intercept is value - slope * maxhyp.
 *
 * Parameters (fp32, GX_TAIL_NPARAM): W1 [256][132], b1 [256], W2 [256][256], b2 [256],
 * W3 [2][256], b3 [2] (row-major, out x in).  norm[4] = mean and scale of the two
 * targets (slope, value); the network works on normalised targets. */
#define GX_TAIL_WINDOW 128
#define GX_TAIL_IN     132
#define GX_TAIL_HIDDEN 256
#define GX_TAIL_OUT    2
#define GX_TAIL_NPARAM (GX_TAIL_HIDDEN * GX_TAIL_IN + GX_TAIL_HIDDEN + GX_TAIL_HIDDEN * GX_TAIL_HIDDEN + \
                        GX_TAIL_HIDDEN + GX_TAIL_OUT * GX_TAIL_HIDDEN + GX_TAIL_OUT)
#define GX_TAIL_MAX_KEEP 512          /* largest subsample drawn by gx_tail_features */
#define GX_STATUS_LEARNED_TAIL 16     /* gx_result.status: e_x, mu, beta come from the model */

typedef struct gx_tail_model gx_tail_model;

/* One feature row: histogram row `query`; keep > 0 subsamples its candidates to `keep`
 * (the top-scoring one always kept, the others drawn without replacement by Floyd's
 * method from a SplitMix64 stream seeded with `seed`); keep = 0 uses them all. */
typedef struct {
    uint32_t query;
    uint32_t keep;
    uint64_t seed;
} gx_tail_sample;

typedef struct {
    float lr, beta1, beta2, eps;  /* Adam */
    float w_slope, w_lgs;         /* loss weights of the two normalised outputs */
} gx_tail_adam;

/* Model with scratch for batches of up to max_batch rows; weights U(+-1/sqrt(fan_in))
 * from std::mt19937_64(seed), biases 0, norm = {0, 1, 0, 1}. */
gx_status gx_tail_model_create(int32_t device, uint32_t max_batch, uint64_t seed, gx_tail_model **out);
gx_status gx_tail_model_free(gx_tail_model *m);
/* Host copies in/out (either pointer may be NULL).  set resets the Adam state; it synchronises. */
gx_status gx_tail_model_set(gx_tail_model *m, const float *params, const float *norm);
gx_status gx_tail_model_get(const gx_tail_model *m, float *params, float *norm, uint64_t *steps);

/* Feature rows for n samples (host array) of the nq queries whose histograms
 * (hist_dev [nq][GX_HIST_BINS]), results (maxhyp), precursor masses and charges (may be
 * NULL: 0) are on the device.  Writes x_dev [n][GX_TAIL_IN] (bf16 bits) and, when not
 * NULL, the subsampled histograms [n][GX_HIST_BINS], their candidate counts and maxhyp.
 * n <= max_batch.  Synchronises the stream. */
gx_status gx_tail_features(gx_tail_model *m, const uint32_t *hist_dev, const gx_result *res_dev,
                           const float *prec_dev, const int32_t *charge_dev, uint32_t nq,
                           const gx_tail_sample *samples_host, uint32_t n, uint16_t *x_dev,
                           uint32_t *sub_hist_dev, int32_t *sub_cpsms_dev, int32_t *hyp_dev, void *stream);
/* Plain FP64 expeRT fit of n histogram rows: fit_dev [n][2] = (slope, intercept). */
gx_status gx_tail_fit_rows(const uint32_t *hist_dev, const int32_t *cpsms_dev, const int32_t *hyp_dev, uint32_t n,
                           double *fit_dev, void *stream);
/* Forward + loss + backward on n rows; targets [n][2] = (slope, value at maxhyp).
 * grad_dev (optional) receives the GX_TAIL_NPARAM gradients, loss_dev (optional) the
 * mean loss.  weights2 (host, optional) = loss weights of the two outputs (default 1, 1). */
gx_status gx_tail_grad(gx_tail_model *m, const uint16_t *x_dev, const float *target_dev, uint32_t n,
                       const float *weights2, float *grad_dev, float *loss_dev, void *stream);
/* Training loss of gx_tail_grad / gx_tail_train_step, per normalised output d = y - t:
 * huber_delta = 0 (the default) the squared error d^2; > 0 Huber's loss, d^2 / (2 delta) for
 * |d| < delta and |d| - delta / 2 beyond.  Huber's loss follows the median of a heavy-tailed
 * target (the full-data fit of a sparse query's histogram varies by orders of magnitude)
 * where the squared error follows its mean. */
gx_status gx_tail_set_loss(gx_tail_model *m, float huber_delta);
/* One Adam step on a batch (gx_tail_grad followed by the update). */
gx_status gx_tail_train_step(gx_tail_model *m, const uint16_t *x_dev, const float *target_dev, uint32_t n,
                             const gx_tail_adam *opt, float *loss_dev, void *stream);
/* pred_dev [n][2] = (slope, log10 survival fraction at maxhyp). */
gx_status gx_tail_predict(gx_tail_model *m, const uint16_t *x_dev, uint32_t n, float *pred_dev, void *stream);
/* Fallback policy over search results on the device: every query with status & 1 and
 * cpsms < sparse_below takes the learned line when it is finite and falling
 * (mu, beta, e_x replaced, status |= GX_STATUS_LEARNED_TAIL, bit 2 re-evaluated against
 * expect_max); all others keep the plain fit.  slope, icpt and e_fp64 keep the plain fit. */
gx_status gx_tail_apply(gx_tail_model *m, const uint32_t *hist_dev, gx_result *res_dev, const float *prec_dev,
                        const int32_t *charge_dev, uint32_t nspec, uint32_t sparse_below, double expect_max,
                        void *stream);
/* Attach a model to a workspace (NULL detaches): every batched search through the
 * workspace (gx_search_host, gx_search_device) then applies the fallback policy of
 * gx_tail_apply with sparse_below after the plain fit, on the workspace's stream or the
 * caller's.  The model must live on the index's device and outlive the attachment. */
gx_status gx_workspace_set_tail(gx_workspace *ws, gx_tail_model *m, uint32_t sparse_below);
/* Synchronises, reports a device-side guard of the model's kernels (GX_ERR_DEVICE_GUARD)
 * and clears it, so that the next check reports only what came after this one. */
gx_status gx_tail_check(gx_tail_model *m);
/* Time limit of each wait of the model's tensor-core kernel for its matrix products, in
 * nanoseconds of the GPU clock (default 1,000,000,000, one second; applies to launches made
 * after the call, process-wide).  A wait that runs out makes the kernel record the guard
 * that gx_tail_check reports, wait (at most one more second) for the product it issued
 * last, free its tensor memory and return without writing its output.  0 makes every
 * wait give up at once: a way to exercise that path.  No counterpart in the reference. */
gx_status gx_tail_set_wait_limit(uint64_t ns);
/* The model's tensor-core GEMM alone: D[M][N] (fp32, row stride ldd) = A * B^T with
 * A(m,k) = a[m*sam + k*sak], B(n,k) = b[n*sbn + k*sbk] (bf16 bits), on the current device. */
gx_status gx_tail_gemm(const uint16_t *a_dev, int64_t sam, int64_t sak, const uint16_t *b_dev, int64_t sbn,
                       int64_t sbk, int32_t M, int32_t N, int32_t K, float *d_dev, int64_t ldd, void *stream);

/* Message of the calling thread's last failure ("" if none). */
const char *gx_last_error(void);
/* Kernel launches issued by this process so far (all gx_* calls). */
uint64_t gx_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* GICOPS_B200_H */
