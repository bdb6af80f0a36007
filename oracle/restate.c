/* Test infrastructure only.  A CPU restatement, in plain C, of the reference's
 * query path; tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it
 * as the checker.  The product never calls it.
 *
 * Each step follows the reference's CPU code (paths relative to the reference
 * project):
 *   window        source/core/dslim_query.cpp:1102-1242 (DSLIM_BinarySearch and its
 *                 BinFindMin/BinFindMax bisections = lower/upper bound on float masses)
 *   bucket probe  source/core/dslim_query.cpp:853-914
 *   scan          source/core/dslim_query.cpp:923-969
 *   hyperscore    lgfact table of source/core/include/utils.h:115-131
 *   top-K         source/core/include/minheap.h:103-271 (insert, increase_key,
 *                 heapify, getMax), capacity from source/core/dslim.cpp:438-444
 *   e-value       source/core/dslim_query.cpp:1017-1061 and
 *                 source/core/expeRT.cpp:396-559 (ModelTailFit), 1149-1201
 *                 (rargmax/argmax/largmax), 1241-1289 (LinearFit)
 * Integer and float types match the reference's (short counts, uint sums,
 * double hyperscore rounded to float, float*10 histogram binning).  Build with
 * -ffp-contract=off so no double operation is fused. */
#include "restate.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int16_t bc, yc;
    uint32_t ibc, iyc;
} byc_t;

void rs_lgfact(double *o)
{
    o[0] = o[1] = log10(1.0);
    for (int i = 2; i < 81; i++) o[i] = log10((double)i) + o[i - 1];
}

/* double -> int as x86-64 cvttsd2si does it: truncation, INT_MIN when NaN or out of range. */
static int32_t to_int_x86(double v)
{
    if (!(v > -2147483649.0 && v < 2147483648.0)) return INT_MIN;
    return (int32_t)v;
}

void rs_window(const rs_length *len, float prec, double dM, int32_t *lo, int32_t *hi)
{
    *lo = 1;
    *hi = 0;
    const int64_t N = len->npep;
    if (dM < 0.0 || N == 0) return;
    const float p1 = (float)((double)prec - dM);
    const float p2 = (float)((double)prec + dM);
    if (p1 != p1 || p2 != p2) return;
    const float *m = len->mass;
    if (p1 > m[N - 1] || p2 < m[0]) return;
    int64_t a = 0, b = N; /* first index with m >= p1 */
    while (a < b) {
        int64_t c = (a + b) >> 1;
        if (m[c] < p1) a = c + 1; else b = c;
    }
    int64_t lo_ = a;
    a = 0; b = N;         /* first index with m > p2 */
    while (a < b) {
        int64_t c = (a + b) >> 1;
        if (p2 < m[c]) b = c; else a = c + 1;
    }
    *lo = (int32_t)lo_;
    *hi = (int32_t)(a - 1);
}

/* ---- minHeap<hCell> ------------------------------------------------------------- */
typedef struct {
    int size, cap;
    rs_cell a[RS_MAXHEAP];
} heap_t;

static void heapify(heap_t *h, int i)
{
    for (;;) {
        int r = (i + 1) * 2, l = r - 1, s = i;
        float sv = h->a[i].hyperscore;
        if (l < h->size && h->a[l].hyperscore < sv) { s = l; sv = h->a[l].hyperscore; }
        if (r < h->size && h->a[r].hyperscore < sv) { s = r; }
        if (s == i) return;
        rs_cell t = h->a[s]; h->a[s] = h->a[i]; h->a[i] = t;
        i = s;
    }
}

static void heap_insert(heap_t *h, const rs_cell *c)
{
    if (h->size == h->cap) {
        if (c->hyperscore < h->a[0].hyperscore) return;   /* increase_key refuses */
        h->a[0] = *c;
        heapify(h, 0);
        return;
    }
    h->a[h->size++] = *c;
    for (int i = (h->size - 1) / 2; i >= 0; i--) heapify(h, i);
}

static rs_cell heap_getmax(const heap_t *h)
{
    if (h->size <= 1) return h->a[0];
    rs_cell m = h->a[h->size - 1];
    for (int k = h->size - 2; k >= h->size / 2; k--)
        if (h->a[k].hyperscore > m.hyperscore) m = h->a[k];
    return m;
}

/* ---- expeRT::ModelTailFit ----------------------------------------------------------- */
static void linear_fit(const double *x, const double *y, int n, double *a, double *b)
{
    if (n == 1) { *a = 0.0; *b = y[0]; return; }
    double xbar = 0.0, ybar = 0.0;
    for (int i = 0; i < n; i++) { xbar = xbar + x[i]; ybar = ybar + y[i]; }
    xbar = xbar / (double)n;
    ybar = ybar / (double)n;
    double top = 0.0, bot = 0.0;
    for (int i = 0; i < n; i++) {
        top = top + (x[i] - xbar) * (y[i] - ybar);
        bot = bot + (x[i] - xbar) * (x[i] - xbar);
    }
    *a = top / bot;
    *b = ybar - *a * xbar;
}

void rs_tailfit(const double *yy, int32_t cpsms, int32_t hyp, rs_result *r)
{
    double mu_t = 0.0, beta_t = 4.0;
    int end1 = hyp - 1;
    for (int p = hyp - 1; p >= 0; p--) if (yy[p] >= 1.0) { end1 = p; break; }
    int stt1 = 0;
    for (int p = 0; p <= end1; p++) if (yy[p] >= 1.0) { stt1 = p; break; }
    if (stt1 == end1) end1 += 1;

    if (cpsms < 1) {
        mu_t = 0.0;
        beta_t = 100.0;
    } else {
        /* sx[1..size] with one slot in front: the reference may read one element
         * before the slice (mark == -1); that slot holds 0 here (the reference reads
         * an allocator header word there, a subnormal that the sums absorb). */
        double buf[RS_HIST + 2];
        double *sx = buf + 1;
        buf[0] = 0.0;
        int size = end1 - stt1 + 1;
        if (size < 0) size = 0;
        double acc = 0.0;
        for (int i = 0; i < size; i++) { acc = acc + yy[stt1 + i]; sx[i] = acc; }
        for (int i = 0; i < size; i++) {
            double v = sx[i] / (double)cpsms;
            v = v + (-1.0);
            sx[i] = -v;
        }
        for (int i = 0; i < size; i++) if (sx[i] > 1.0) sx[i] = 0.999;
        if (size > 0) {
            int rep = size - 1;
            for (int p = size - 1; p >= 0; p--) if (sx[p] >= 1e-4) { rep = p; break; }
            const double v = sx[rep];
            for (int i = 0; i < size; i++) if (sx[i] <= 0.0) sx[i] = v;
        }
        for (int i = 0; i < size; i++) sx[i] = log10(sx[i]);

        int mark = 0, mark2 = 0;
        if (size >= 3) {
            const double hgt = sx[size - 1] - sx[0];
            const double t22 = sx[0] + hgt * 0.22;
            int lm = 0;
            for (int p = 0; p <= size - 1; p++) if (sx[p] <= t22) { lm = p; break; }
            mark = lm - 1;
            if (size > 3) {
                const double t87 = sx[0] + hgt * 0.87;
                mark2 = size - 1;
                for (int p = size - 1; p >= 0; p--) if (sx[p] >= t87) { mark2 = p; break; }
                if (mark2 == size) mark2 -= 1;
            } else {
                mark2 = size - 1;
            }
            if (mark >= mark2) mark = mark2 - 1;
        } else {
            mark = 0;
            mark2 = size - 1;
        }
        const int n = mark2 - mark + 1;
        double X[RS_HIST + 2];
        for (int i = 0; i < n; i++) X[i] = (double)(stt1 + mark + i);
        if (n >= 1) {
            linear_fit(X, sx + mark, n, &mu_t, &beta_t);
        } else {
            mu_t = NAN;   /* 0/0 in the reference's LinearFit */
            beta_t = NAN;
        }
    }
    r->slope = mu_t;
    r->icpt = beta_t;
    r->mu = to_int_x86(mu_t * 1e6);
    r->beta = to_int_x86(beta_t * 1e6);
    r->stt1 = stt1;
    r->end1 = end1;
    double w = (double)r->mu, b = (double)r->beta;
    w /= 1e6;
    b /= 1e6;
    const double lgs = (w * (double)hyp) + b;
    r->e_x = pow(10.0, lgs) * (double)(uint32_t)cpsms;
    r->e_fp64 = pow(10.0, mu_t * (double)hyp + beta_t) * (double)(uint32_t)cpsms;
}

/* ---- one spectrum ------------------------------------------------------------------ */
static int peak_ok(int32_t qion, const rs_params *par)
{
    const double upper = (par->max_mass * (double)par->scale) - 1.0 - (double)par->dF;
    return qion > (int32_t)par->dF && (double)qion < upper;
}

static void search_one(const rs_length *lens, int nlen, const int32_t *moz, const int32_t *intn, int npk,
                       float prec, double dM, const rs_params *par, const double *lgf, byc_t *byc,
                       rs_result *res, uint32_t *hist)
{
    double surv[RS_HIST];
    memset(surv, 0, sizeof(surv));
    heap_t heap;
    memset(&heap, 0, sizeof(heap));
    heap.cap = par->heap_cap;
    uint32_t cpsms = 0;
    int status = 0;

    for (int ixx = 0; ixx < nlen; ixx++) {
        const rs_length *ln = lens + ixx;
        const uint32_t speclen = ln->speclen, half = speclen / 2;
        int32_t lo, hi;
        rs_window(ln, prec, dM, &lo, &hi);
        if (hi < lo) continue;
        const uint32_t idlo = (uint32_t)lo * speclen;
        const uint32_t idhi = ((uint32_t)(hi + 1) * speclen) - 1;
        for (int k = 0; k < npk; k++) {
            const int32_t q = moz[k];
            const uint32_t in = (uint32_t)intn[k];
            if (!peak_ok(q, par)) continue;
            for (uint32_t bin = (uint32_t)q - par->dF; bin < (uint32_t)q + 1 + par->dF; bin++) {
                const uint32_t s = ln->bA[bin], e = ln->bA[bin + 1];
                if (e - s < 1) continue;
                uint32_t a = s, b = e;
                while (a < b) { uint32_t c = a + ((b - a) >> 1); if (ln->iA[c] < idlo) a = c + 1; else b = c; }
                const uint32_t st = a;
                b = e;
                while (a < b) { uint32_t c = a + ((b - a) >> 1); if (idhi < ln->iA[c]) b = c; else a = c + 1; }
                for (uint32_t ion = st; ion < a; ion++) {
                    const uint32_t raw = ln->iA[ion];
                    const uint32_t pp = raw / speclen;
                    const uint32_t isY = (raw % speclen) / half;
                    const uint32_t isB = 1 - isY;
                    byc_t *el = byc + pp;
                    el->bc = (int16_t)(el->bc + (int16_t)isB);
                    el->ibc += in * isB;
                    el->yc = (int16_t)(el->yc + (int16_t)isY);
                    el->iyc += in * isY;
                }
            }
        }
        for (int32_t it = lo; it <= hi; it++) {
            const uint16_t bcc = (uint16_t)byc[it].bc, ycc = (uint16_t)byc[it].yc;
            const uint16_t shpk = (uint16_t)(bcc + ycc);
            if (shpk >= par->min_shp) {
                int bi = bcc, yi = ycc;
                if (bi > 80 || yi > 80) { status |= 4; if (bi > 80) bi = 80; if (yi > 80) yi = 80; }
                const double h1 = lgf[bi] + lgf[yi];
                float h = (float)(h1 + log10((double)(uint32_t)(1u + byc[it].ibc)) +
                                  log10((double)(uint32_t)(1u + byc[it].iyc)) - 4);
                if (h > 0) {
                    if (h >= 80) h = 79;
                    rs_cell c;
                    c.hyperscore = h;
                    c.psid = it;
                    c.idxoffset = (uint16_t)ixx;
                    c.sharedions = shpk;
                    c.totalions = (uint16_t)speclen;
                    c.pad = 0;
                    heap_insert(&heap, &c);
                    cpsms += 1;
                    surv[(int)((double)(h * 10.0f) + 0.5)] += 1;
                }
            }
        }
        memset(byc + lo, 0, sizeof(byc_t) * (size_t)(hi - lo + 1));
    }

    memset(res, 0, sizeof(*res));
    res->cpsms = (int32_t)cpsms;
    res->heap_size = heap.size;
    memcpy(res->heap, heap.a, sizeof(rs_cell) * (size_t)heap.size);
    if (cpsms > 0 && cpsms >= par->min_cpsm) {   /* min_cpsm 0 acts as 1: an empty heap has no top */
        status |= 1;
        res->top = heap_getmax(&heap);
        res->maxhyp = (int32_t)((double)(res->top.hyperscore * 10.0f) + 0.5);
        rs_tailfit(surv, (int32_t)cpsms, res->maxhyp, res);
        if (res->e_x < par->expect_max) status |= 2;
    }
    res->status = status;
    if (hist)
        for (int i = 0; i < RS_HIST; i++) hist[i] = (uint32_t)surv[i];
}

static uint32_t max_npep(const rs_length *lens, int nlen)
{
    uint32_t m = 1;
    for (int i = 0; i < nlen; i++) if (lens[i].npep > m) m = lens[i].npep;
    return m;
}

int rs_search(const rs_length *lens, int nlen, const uint32_t *qidx, const int32_t *moz, const int32_t *intn,
              const float *prec, const double *dMq, int nspec, const rs_params *par, rs_result *out,
              uint32_t *hist, int nthreads)
{
    if (par->heap_cap < 1 || par->heap_cap > RS_MAXHEAP) return -1;
    double lgf[81];
    rs_lgfact(lgf);
    const uint32_t mx = max_npep(lens, nlen);
    int err = 0;
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
    {
        byc_t *byc = (byc_t *)calloc(mx, sizeof(byc_t));
        if (!byc) {
#pragma omp atomic write
            err = -2;
        }
#pragma omp for schedule(dynamic, 4)
        for (int q = 0; q < nspec; q++) {
            if (!byc) continue;
            const uint32_t a = qidx[q], b = qidx[q + 1];
            const double dM = dMq ? dMq[q] : par->dM;
            search_one(lens, nlen, moz + a, intn + a, (int)(b - a), prec[q], dM, par, lgf, byc, out + q,
                       hist ? hist + (size_t)q * RS_HIST : NULL);
        }
        free(byc);
    }
    return err;
}

int64_t rs_candidates(const rs_length *lens, int nlen, const int32_t *moz, const int32_t *intn, int npk,
                      float prec, double dM, const rs_params *par, rs_cand *out, int64_t cap)
{
    double lgf[81];
    rs_lgfact(lgf);
    byc_t *byc = (byc_t *)calloc(max_npep(lens, nlen), sizeof(byc_t));
    if (!byc) return -1;
    int64_t n = 0;
    for (int ixx = 0; ixx < nlen; ixx++) {
        const rs_length *ln = lens + ixx;
        const uint32_t speclen = ln->speclen, half = speclen / 2;
        int32_t lo, hi;
        rs_window(ln, prec, dM, &lo, &hi);
        if (hi < lo) continue;
        const uint32_t idlo = (uint32_t)lo * speclen, idhi = ((uint32_t)(hi + 1) * speclen) - 1;
        for (int k = 0; k < npk; k++) {
            const int32_t q = moz[k];
            if (!peak_ok(q, par)) continue;
            for (uint32_t bin = (uint32_t)q - par->dF; bin < (uint32_t)q + 1 + par->dF; bin++)
                for (uint32_t ion = ln->bA[bin]; ion < ln->bA[bin + 1]; ion++) {
                    const uint32_t raw = ln->iA[ion];
                    if (raw < idlo || raw > idhi) continue;
                    const uint32_t isY = (raw % speclen) / half;
                    byc_t *el = byc + raw / speclen;
                    el->bc = (int16_t)(el->bc + (int16_t)(1 - isY));
                    el->yc = (int16_t)(el->yc + (int16_t)isY);
                    el->ibc += (uint32_t)intn[k] * (1 - isY);
                    el->iyc += (uint32_t)intn[k] * isY;
                }
        }
        for (int32_t it = lo; it <= hi; it++) {
            const byc_t *e = byc + it;
            if (e->bc == 0 && e->yc == 0) continue;
            if (n < cap) {
                rs_cand *c = out + n;
                c->ixx = (uint16_t)ixx;
                c->bc = (uint16_t)e->bc;
                c->yc = (uint16_t)e->yc;
                c->pad = 0;
                c->psid = it;
                c->ibc = e->ibc;
                c->iyc = e->iyc;
                c->h = 0.0f;
                const uint16_t shpk = (uint16_t)((uint16_t)e->bc + (uint16_t)e->yc);
                if (shpk >= par->min_shp) {
                    int bi = (uint16_t)e->bc > 80 ? 80 : (uint16_t)e->bc, yi = (uint16_t)e->yc > 80 ? 80 : (uint16_t)e->yc;
                    float h = (float)(lgf[bi] + lgf[yi] + log10((double)(uint32_t)(1u + e->ibc)) +
                                      log10((double)(uint32_t)(1u + e->iyc)) - 4);
                    if (h > 0) c->h = h >= 80 ? 79.0f : h;
                }
            }
            n++;
        }
        memset(byc + lo, 0, sizeof(byc_t) * (size_t)(hi - lo + 1));
    }
    free(byc);
    return n;
}

void rs_traffic(const rs_length *lens, int nlen, const int32_t *moz, int npk, float prec, double dM,
                const rs_params *par, int64_t *ids, int64_t *bins)
{
    int64_t ni = 0, nb = 0;
    uint32_t *seen = NULL;
    int nseen = 0, capseen = 0;
    for (int ixx = 0; ixx < nlen; ixx++) {
        const rs_length *ln = lens + ixx;
        int32_t lo, hi;
        rs_window(ln, prec, dM, &lo, &hi);
        if (hi < lo) continue;
        const uint32_t idlo = (uint32_t)lo * ln->speclen, idhi = ((uint32_t)(hi + 1) * ln->speclen) - 1;
        nseen = 0;
        for (int k = 0; k < npk; k++) {
            if (!peak_ok(moz[k], par)) continue;
            for (uint32_t bin = (uint32_t)moz[k] - par->dF; bin < (uint32_t)moz[k] + 1 + par->dF; bin++) {
                int dup = 0;
                for (int j = 0; j < nseen; j++) if (seen[j] == bin) { dup = 1; break; }
                if (dup) continue;
                if (nseen == capseen) {
                    capseen = capseen ? 2 * capseen : 2048;
                    seen = (uint32_t *)realloc(seen, sizeof(uint32_t) * (size_t)capseen);
                }
                seen[nseen++] = bin;
                nb++;
                for (uint32_t ion = ln->bA[bin]; ion < ln->bA[bin + 1]; ion++)
                    if (ln->iA[ion] >= idlo && ln->iA[ion] <= idhi) ni++;
            }
        }
    }
    free(seen);
    *ids = ni;
    *bins = nb;
}

/* ---- query preprocessing: peak picking and intensity normalisation -------------------
 * source/core/msquery.cpp:338-423 (MSQuery::pickpeaks, the form the MS2 -> .pbin
 * conversion uses) with the key-value quicksort of source/core/include/keyval.h:49-129
 * (Hoare partition around the middle element; its OpenMP tasks only split disjoint
 * ranges, so the result is that of the serial recursion). */

/* double -> int32 as x86's truncating conversion does it: out-of-range and NaN give
 * INT32_MIN (the reference converts with an implicit int cast). */
int32_t rs_cvt_i32(double v)
{
    return (v >= -2147483648.0 && v < 2147483648.0) ? (int32_t)v : INT32_MIN;
}

static void kv_sort(int32_t *key, int32_t *val, long left, long right)
{
    long i = left, j = right;
    const int32_t pivot = key[(left + right) / 2];
    while (i <= j) {
        while (key[i] < pivot) i++;
        while (key[j] > pivot) j--;
        if (i <= j) {
            const int32_t tk = key[i], tv = val[i];
            key[i] = key[j];
            val[i] = val[j];
            key[j] = tk;
            val[j] = tv;
            i++;
            j--;
        }
    }
    if (left < j) kv_sort(key, val, left, j);
    if (i < right) kv_sort(key, val, i, right);
}

/* One spectrum: mz/in hold the n_vec values collected since the previous spectrum
 * (n_vec == specsize except for peaks before a file's first S line); the first specsize
 * are sorted by intensity and scaled in place.  Returns the number of peaks kept: the
 * last `kept` values of the arrays. */
int rs_pickpeaks(int32_t *mz, int32_t *in, int n_vec, int specsize, int32_t base_int, int32_t min_int, int qalen)
{
    (void)n_vec;
    if (specsize <= 0) return 0;
    kv_sort(in, mz, 0, specsize - 1);
    const double factor = (double)base_int / (double)in[specsize - 1];
    in[specsize - 1] = base_int;
    int kept = 1;
    for (int j = specsize - 2; j >= specsize - qalen && j >= 0; j--) {
        in[j] = rs_cvt_i32((double)in[j] * factor);
        if (in[j] >= min_int)
            kept++;
        else
            break;
    }
    return kept >= qalen ? qalen : kept;
}
