/* Test infrastructure only: CPU restatement of the reference's query path.
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
 * checker; never by the product.  See restate.c for the reference lines each
 * step follows. */
#ifndef GX_RESTATE_H
#define GX_RESTATE_H

#include <stdint.h>

#define RS_HIST 802      /* 2 + MAX_HYPERSCORE*10 */
#define RS_MAXHEAP 63

typedef struct {
    uint32_t peplen;     /* L */
    uint32_t npep;       /* number of index entries N */
    uint32_t speclen;    /* 2*(L-1)*maxz */
    const float *mass;   /* [N] sorted precursor masses */
    const uint32_t *bA;  /* [nbins] CSR row offsets (per 0.01 Da bin) */
    const uint32_t *iA;  /* [N*speclen] ion ids, ascending within a bin */
} rs_length;

typedef struct {
    double dM;           /* precursor tolerance (Da); per-query values override */
    uint32_t dF;         /* fragment tolerance in bins */
    uint32_t scale;      /* bins per Da (100) */
    double max_mass;     /* 5000 */
    uint32_t min_shp;    /* 4 */
    uint32_t min_cpsm;   /* 4 */
    int32_t heap_cap;    /* (1 << ceil-ish log2(topmatches)) - 1, e.g. 7 */
    double expect_max;   /* PSMs with e >= expect_max are not printed */
} rs_params;

typedef struct {
    float hyperscore;
    int32_t psid;
    uint16_t idxoffset;
    uint16_t sharedions;
    uint16_t totalions;
    uint16_t pad;
} rs_cell;

typedef struct {
    int32_t cpsms;       /* candidates with shp >= min_shp and h > 0 */
    int32_t status;      /* bit0: cpsms >= min_cpsm (tail fit run), bit1: e < expect_max (printed),
                            bit2: an index read lgfact past its end (bc or yc > 80) */
    rs_cell top;         /* minHeap::getMax() */
    int32_t maxhyp;      /* (int)(top.h*10+0.5) */
    int32_t mu, beta;    /* tail fit slope/intercept x1e6, truncated to int */
    int32_t stt1, end1;  /* curve region */
    double slope, icpt;  /* unquantized FP64 fit */
    double e_x;          /* the reference's e-value (quantized slope/intercept) */
    double e_fp64;       /* e-value from the unquantized fit */
    int32_t heap_size;
    int32_t pad2;
    rs_cell heap[RS_MAXHEAP];  /* final heap array, in heap order */
} rs_result;

/* One detailed candidate record (for tests of the scorecard). */
typedef struct {
    uint16_t ixx;
    uint16_t bc, yc;
    uint16_t pad;
    int32_t psid;
    uint32_t ibc, iyc;
    float h;             /* 0 if not a candidate PSM */
} rs_cand;

#ifdef __cplusplus
extern "C" {
#endif

/* Hyperscore table lgfact[i] = sum_{k<=i} log10(k), 81 entries. */
void rs_lgfact(double *out81);

/* Search nspec spectra.  qidx: [nspec+1] CSR offsets into moz/intn.  dMq may be
 * NULL (use par->dM) or per-query tolerances in Da.  hist (optional) receives
 * RS_HIST counts per spectrum.  Returns 0 on success. */
int rs_search(const rs_length *lens, int nlen, const uint32_t *qidx, const int32_t *moz,
              const int32_t *intn, const float *prec, const double *dMq, int nspec,
              const rs_params *par, rs_result *out, uint32_t *hist, int nthreads);

/* Window [lo, hi] of one precursor over one length (lo > hi: skipped). */
void rs_window(const rs_length *len, float prec, double dM, int32_t *lo, int32_t *hi);

/* Every scorecard entry with bc+yc > 0 of one spectrum, in (ixx, psid) order.
 * Returns the number of records (written up to cap). */
int64_t rs_candidates(const rs_length *lens, int nlen, const int32_t *moz, const int32_t *intn,
                      int npk, float prec, double dM, const rs_params *par, rs_cand *out, int64_t cap);

/* Tail fit of one histogram (expeRT::ModelTailFit); fills mu..e_fp64 of r. */
void rs_tailfit(const double *hist802, int32_t cpsms, int32_t maxhyp, rs_result *r);

/* Scan-over-candidates reference count of in-window ion ids read (4 B each, once per
 * distinct probed bin) and distinct probed bins, summed over lengths: the
 * algorithmic-traffic figures of the roofline. */
void rs_traffic(const rs_length *lens, int nlen, const int32_t *moz, int npk, float prec, double dM,
                const rs_params *par, int64_t *ids, int64_t *bins);

/* Query preprocessing (source/core/msquery.cpp:338-423, keyval.h:49-129). */
int32_t rs_cvt_i32(double v);
int rs_pickpeaks(int32_t *mz, int32_t *in, int n_vec, int specsize, int32_t base_int, int32_t min_int, int qalen);

#ifdef __cplusplus
}
#endif

#endif
