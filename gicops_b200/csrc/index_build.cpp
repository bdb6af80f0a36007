// Host-side index builder: peptide sequences of one length -> entries sorted by
// precursor mass -> CSR fragment-ion index (bA row offsets per 0.01 Da bin, iA ion
// ids ascending within a bin).  It produces exactly the arrays the reference's
// CPU build produces, so that an index built here and one built by the reference
// are interchangeable (paths relative to the reference project):
//   mass filter           source/core/lbe_internal.cpp:398-498, utils.cpp:240-252
//   variant enumeration   source/core/mods.cpp:273-324 (depth-first: modify, then skip),
//                         per-peptide ordering mods.cpp:101-118 + slm_dsts.h:191-271
//   variant mass          source/core/utils.cpp:306-331 (only the first modification's
//                         mass is added: the loop's shift count is the mask itself)
//   mass sort             source/core/lbe_internal.cpp:189 (std::sort on mass)
//   fragment ions         source/core/utils.cpp:161-226, 347-474 (float arithmetic)
//   CSR                   source/core/dslim.cpp:231-402, 474-504 (bins clamped to the last bin,
//                         out-of-range entries put all ions in bin 0)
// The per-peptide variant order and the mass sort use the C library's qsort and
// libstdc++'s std::sort with comparators equivalent to the reference's, so entries of
// equal mass land in the same order as in the reference's index.

#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_internal.h"
#include "gx_ions.h"

namespace {

using gx::ions::IonTables;
using gx::ions::kMaxModTypes;
using gx::ions::kMaxSeqLen;

struct ModTable {
    int cond_of[256];            // residue -> modification type, -1 if none
    int limit;                   // modified residues per peptide
    std::vector<int> per_type;   // per-type limits
    IonTables t;                 // residue tables, (uint)(mass*scale) per modification, scale
};

void enumerate_variants(const char *seq, int L, std::vector<int> &left, int total, const gx_pep_entry &cont,
                        int letter, bool novel, int seen, uint32_t refid, const ModTable &mt,
                        std::vector<gx_pep_entry> &out)
{
    if (novel && letter != 0) {
        gx_pep_entry e = cont;
        e.mass = gx::ions::mod_mass_first_only(mt.t, seq, (unsigned)L, e.modnum);
        out.push_back(e);
    }
    if (total == 0 || letter >= L) return;
    const int c = mt.cond_of[(unsigned char)seq[letter]];
    if (c != -1 && left[c] > 0) {
        gx_pep_entry d = cont;
        d.sites |= (uint64_t)1 << letter;
        d.modnum += (uint32_t)((1 << (4 * seen)) * (1 + c));
        d.seqid = refid;
        left[c] -= 1;
        enumerate_variants(seq, L, left, total - 1, d, letter + 1, true, seen + 1, refid, mt, out);
        left[c] += 1;
    }
    enumerate_variants(seq, L, left, total, cont, letter + 1, false, seen, refid, mt, out);
}

// Distance marks of a site mask: first set bit from the N-terminus (s1) and last set
// bit scanning back from MAX_SEQ_LEN (s3), with the reference's loop semantics.
int span_key(uint64_t sites)
{
    int s1 = 0;
    while (((sites >> s1) & 1u) != 1u && s1++ < kMaxSeqLen) {
    }
    int s3 = kMaxSeqLen;
    while (((sites >> s3) & 1u) != 1u && s3-- > s1) {
    }
    return s1 + kMaxSeqLen - s3;
}

int cmp_variants(const void *l, const void *r)
{
    const int a = span_key(((const gx_pep_entry *)l)->sites);
    const int b = span_key(((const gx_pep_entry *)r)->sites);
    if (a < b) return 1;
    if (a > b) return -1;
    return 0;
}

}  // namespace

struct gx_host_length {
    uint32_t L = 0, maxz = 0, speclen = 0, nbins = 0;
    std::vector<char> seqs;             // kept peptides, npep_kept x L
    std::vector<gx_pep_entry> entries;  // mass-sorted
    std::vector<float> mass;
    std::vector<uint32_t> bA, iA;
};

namespace {

// Steps 1-2 of a build: mass filter, variant enumeration, mass sort (into h).
gx_status build_entries(const char *seqs, uint32_t npep, uint32_t L, const gx_build_params *bp, gx_host_length **out,
                        ModTable &mt)
{
    using namespace gx;
    if (!out || !bp || (!seqs && npep)) return fail(GX_ERR_INVLD_PTR, "gx_build_length: null argument");
    *out = nullptr;
    if (L < 2 || L > (uint32_t)kMaxSeqLen || bp->maxz < 1 || bp->maxz > 6 || bp->scale == 0 ||
        bp->nmods > (uint32_t)kMaxModTypes || bp->max_mass <= bp->min_mass)
        return fail(GX_ERR_INVLD_PARAM, "gx_build_length: bad parameters");
    const int threads = bp->threads > 0 ? bp->threads : omp_get_max_threads();

    for (int &c : mt.cond_of) c = -1;
    mt.limit = (int)bp->mods_per_pep;
    mt.t = gx::ion_tables(bp);
    for (uint32_t i = 0; i < bp->nmods; i++) {
        for (int j = 0; j < 4 && bp->mods[i].residues[j]; j++)
            mt.cond_of[(unsigned char)bp->mods[i].residues[j]] = (int)i;
        mt.per_type.push_back((int)bp->mods[i].max_per_pep);
    }
    for (uint64_t i = 0; i < (uint64_t)npep * L; i++)
        if (seqs[i] < 'A' || seqs[i] > 'Z') return fail(GX_ERR_INVLD_PARAM, "gx_build_length: non-letter residue");

    auto *h = new (std::nothrow) gx_host_length();
    if (!h) return fail(GX_ERR_BAD_MEM_ALLOC, "gx_build_length: out of host memory");
    h->L = L;
    h->maxz = bp->maxz;
    h->speclen = 2 * (L - 1) * bp->maxz;
    h->nbins = bp->max_mass * bp->scale + 1;

    // 1. mass filter (kept in file order)
    std::vector<uint32_t> kept;
    std::vector<float> kmass;
    for (uint32_t i = 0; i < npep; i++) {
        const float m = gx::ions::pep_mass(mt.t, seqs + (size_t)i * L, L);
        if (m >= (float)bp->min_mass && m <= (float)bp->max_mass) {
            kept.push_back(i);
            kmass.push_back(m);
        }
    }
    const uint32_t np = (uint32_t)kept.size();
    h->seqs.resize((size_t)np * L);
    for (uint32_t i = 0; i < np; i++) std::memcpy(&h->seqs[(size_t)i * L], seqs + (size_t)kept[i] * L, L);

    // 2. entries: peptides, then each peptide's variants (ordered per peptide)
    std::vector<std::vector<gx_pep_entry>> var(np);
    if (mt.limit > 0 && bp->nmods > 0) {
#pragma omp parallel for num_threads(threads) schedule(dynamic, 256)
        for (int64_t i = 0; i < (int64_t)np; i++) {
            std::vector<int> left = mt.per_type;
            gx_pep_entry root{};
            enumerate_variants(&h->seqs[(size_t)i * L], (int)L, left, mt.limit, root, 0, false, 0, (uint32_t)i, mt,
                               var[i]);
            if (var[i].size() > 1) std::qsort(var[i].data(), var[i].size(), sizeof(gx_pep_entry), cmp_variants);
        }
    }
    size_t nvar = 0;
    for (auto &v : var) nvar += v.size();
    const uint64_t N = (uint64_t)np + nvar;
    if (N * h->speclen >= (1ull << 32) || N >= (1ull << 31)) {
        delete h;
        return fail(GX_ERR_INVLD_SIZE, "gx_build_length: more than 2^32 ion ids in one length");
    }
    h->entries.resize(N);
    for (uint32_t i = 0; i < np; i++) h->entries[i] = gx_pep_entry{kmass[i], i, 0, 0, 0};
    size_t w = np;
    for (auto &v : var) {
        std::copy(v.begin(), v.end(), h->entries.begin() + w);
        w += v.size();
        std::vector<gx_pep_entry>().swap(v);
    }
    std::sort(h->entries.begin(), h->entries.end(),
              [](const gx_pep_entry &a, const gx_pep_entry &b) { return a.mass < b.mass; });
    h->mass.resize(N);
    for (uint64_t k = 0; k < N; k++) h->mass[k] = h->entries[k].mass;
    *out = h;
    return GX_SUCCESS;
}

}  // namespace

extern "C" gx_status gx_build_length_entries(const char *seqs, uint32_t npep, uint32_t L, const gx_build_params *bp,
                                             gx_host_length **out)
{
    ModTable mt;
    return build_entries(seqs, npep, L, bp, out, mt);
}

extern "C" gx_status gx_build_length(const char *seqs, uint32_t npep, uint32_t L, const gx_build_params *bp,
                                     gx_host_length **out)
{
    ModTable mt;
    gx_host_length *h = nullptr;
    const gx_status st = build_entries(seqs, npep, L, bp, &h, mt);
    if (st != GX_SUCCESS) return st;
    const int threads = bp->threads > 0 ? bp->threads : omp_get_max_threads();
    const uint64_t N = h->entries.size();

    // 3. fragment ions -> bins; 4. stable counting sort by bin
    const uint32_t speclen = h->speclen;
    const uint32_t topbin = bp->max_mass * bp->scale;  // bins >= topbin are clamped to topbin-1
    std::vector<uint32_t> bins((size_t)N * speclen);
    const int T = std::max(1, std::min<int>(threads, (int)((N + 4095) / 4096)));
    std::vector<std::vector<uint32_t>> cnt(T, std::vector<uint32_t>(topbin + 1, 0));
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const uint64_t k0 = N * t / T, k1 = N * (t + 1) / T;
        uint32_t *c = cnt[t].data();
        const uint32_t n1 = L - 1;
        for (uint64_t k = k0; k < k1; k++) {
            const gx_pep_entry &e = h->entries[k];
            const char *seq = &h->seqs[(size_t)e.seqid * L];
            uint32_t *dst = &bins[(size_t)k * speclen];
            if (gx::ions::entry_binned(mt.t, seq, L, e.sites, e.modnum, (double)bp->min_mass, (double)bp->max_mass)) {
                // positions: b ions of charge z at z*(L-1), y ions at (maxz + z)*(L-1)
                for (uint32_t z = 0; z < bp->maxz; z++) {
                    gx::ions::ion_series(mt.t, seq, L, e.sites, e.modnum, z, false, topbin, dst + z * n1);
                    gx::ions::ion_series(mt.t, seq, L, e.sites, e.modnum, z, true, topbin, dst + (bp->maxz + z) * n1);
                }
                for (uint32_t ion = 0; ion < speclen; ion++) c[dst[ion]]++;
            } else {
                std::memset(dst, 0, sizeof(uint32_t) * speclen);
                c[0] += speclen;
            }
        }
    }
    h->bA.assign((size_t)h->nbins, 0);
    {
        uint64_t run = 0;
        for (uint32_t b = 0; b < topbin; b++) {
            h->bA[b] = (uint32_t)run;
            uint64_t tot = 0;
            for (int t = 0; t < T; t++) {
                const uint32_t v = cnt[t][b];
                cnt[t][b] = (uint32_t)(run + tot);  // thread t's first slot in bin b
                tot += v;
            }
            run += tot;
        }
        for (uint32_t b = topbin; b < h->nbins; b++) h->bA[b] = (uint32_t)run;
    }
    h->iA.resize((size_t)N * speclen);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num();
        const uint64_t k0 = N * t / T, k1 = N * (t + 1) / T;
        uint32_t *c = cnt[t].data();
        for (uint64_t id = k0 * speclen; id < k1 * speclen; id++) h->iA[c[bins[id]]++] = (uint32_t)id;
    }
    *out = h;
    return GX_SUCCESS;
}

extern "C" gx_status gx_host_length_desc(const gx_host_length *h, gx_length_desc *d)
{
    if (!h || !d) return gx::fail(GX_ERR_INVLD_PTR, "gx_host_length_desc: null argument");
    d->peplen = h->L;
    d->npep = (uint32_t)h->entries.size();
    d->speclen = h->speclen;
    d->pad = 0;
    d->mass = h->mass.data();
    d->bA = h->bA.empty() ? nullptr : h->bA.data();   // entries-only lengths have no CSR
    d->iA = h->iA.empty() ? nullptr : h->iA.data();
    return GX_SUCCESS;
}

extern "C" const gx_pep_entry *gx_host_length_entries(const gx_host_length *h)
{
    return h ? h->entries.data() : nullptr;
}

extern "C" const char *gx_host_length_seqs(const gx_host_length *h, uint32_t *npep_kept)
{
    if (!h) return nullptr;
    if (npep_kept) *npep_kept = (uint32_t)(h->seqs.size() / (h->L ? h->L : 1));
    return h->seqs.data();
}

extern "C" void gx_host_length_free(gx_host_length *h) { delete h; }
