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

namespace {

constexpr int kMaxSeqLen = 60;
constexpr int kMaxModTypes = 15;

// Residue masses and the fixed carbamidomethyl C (cmake/Templates/aamasses.hpp.in:25-80):
// double literals narrowed to float, as the reference's constexpr float tables are.
constexpr double kNAA = -20000.0;
const float kAAMass[26] = {
    (float)71.03712, (float)kNAA, (float)103.00919, (float)115.030, (float)129.0426, (float)147.068,
    (float)57.02146, (float)137.060, (float)113.084, (float)kNAA, (float)128.094, (float)113.084,
    (float)131.0405, (float)114.043, (float)kNAA, (float)97.0527, (float)128.05858, (float)156.1012,
    (float)87.032, (float)101.0476, (float)kNAA, (float)99.06841, (float)186.0793, (float)kNAA,
    (float)163.0633, (float)kNAA};
const float kStatMod[26] = {0, 0, (float)57.021464, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                            0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
constexpr float kH2O = 18.015f;
constexpr float kProton = 1.00727647f;

inline int aa(char c) { return c - 'A'; }
inline float aa_z(char c, unsigned z) { return (kAAMass[aa(c)] + kStatMod[aa(c)]) + (kProton * (float)z); }

float pep_mass(const char *s, unsigned L)
{
    float m = kH2O;
    for (unsigned l = 0; l < L; l++) m += kAAMass[aa(s[l])] + kStatMod[aa(s[l])];
    return m;
}

struct ModTable {
    int cond_of[256];            // residue -> modification type, -1 if none
    int limit;                   // modified residues per peptide
    std::vector<int> per_type;   // per-type limits
    uint32_t mod_mass[kMaxModTypes];  // (uint)(mass*scale)
    unsigned scale;
};

float mod_mass_first_only(const char *s, unsigned L, uint32_t modnum, const ModTable &mt)
{
    float m = kH2O;
    for (unsigned l = 0; l < L; l++) {
        m += kAAMass[aa(s[l])];
        m += kStatMod[aa(s[l])];
    }
    // The reference's loop shifts by the mask (0xF0), which x86 reduces mod 32 to
    // 16, so its second pass always reads 0: exactly one modification contributes.
    const uint32_t first = modnum & 0x0Fu;
    if (first != 0) m += ((float)mt.mod_mass[first - 1]) / (float)mt.scale;
    return m;
}

void enumerate_variants(const char *seq, int L, std::vector<int> &left, int total, const gx_pep_entry &cont,
                        int letter, bool novel, int seen, uint32_t refid, const ModTable &mt,
                        std::vector<gx_pep_entry> &out)
{
    if (novel && letter != 0) {
        gx_pep_entry e = cont;
        e.mass = mod_mass_first_only(seq, (unsigned)L, e.modnum, mt);
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

// Theoretical spectrum (bins) of one entry into spec[speclen]; returns its mass.
float entry_spectrum(const char *seq, unsigned L, const gx_pep_entry &e, unsigned maxz, double minmass,
                     double maxmass, const ModTable &mt, std::vector<float> &f, uint32_t *spec, bool *filled)
{
    const unsigned scale = mt.scale;
    const unsigned n1 = L - 1;
    *filled = false;
    float mass;
    if (e.modnum == 0) {
        mass = pep_mass(seq, L);
        if (!(mass > 0)) return mass;
    } else {
        if (e.sites == 0) return (float)kNAA;
        mass = mod_mass_first_only(seq, L, e.modnum, mt);
        if (!(mass > minmass && mass < maxmass)) return mass;
    }
    f.assign((size_t)2 * maxz * n1, 0.0f);
    for (unsigned z = 0; z < maxz; z++) {
        const unsigned bs = z * n1, ys = z * n1 + maxz * n1;
        f[bs] = aa_z(seq[0], z + 1);
        f[ys] = aa_z(seq[L - 1], z + 1) + kH2O;
        for (unsigned l = 1; l < n1; l++) {
            f[bs + l] = f[bs + l - 1] + aa_z(seq[l], 0);
            f[ys + l] = f[ys + l - 1] + aa_z(seq[L - 1 - l], 0);
        }
    }
    if (e.modnum == 0) {
        for (unsigned z = 0; z < maxz; z++) {
            const unsigned bs = z * n1, ys = z * n1 + maxz * n1;
            for (unsigned l = 0; l < n1; l++) {
                spec[bs + l] = (uint32_t)((f[bs + l] * (float)scale) / (float)(z + 1));
                spec[ys + l] = (uint32_t)((f[ys + l] * (float)scale) / (float)(z + 1));
            }
        }
    } else {
        int nums[kMaxModTypes];
        int seen = 0;
        uint32_t mask = e.modnum;
        for (int i = 0; i < kMaxModTypes; i++) {
            nums[i] = (int)(mask & 0x0Fu) - 1;
            mask /= 16;
            if (nums[i] != -1) seen++;
        }
        char pos[kMaxSeqLen + 2];
        for (unsigned i = 0; i < L; i++) pos[i] = ((e.sites >> i) & 1u) ? 1 : 0;
        for (unsigned z = 0; z < maxz; z++) {
            const unsigned bs = z * n1;
            unsigned cnt = 0;
            for (unsigned l = 0; l < n1; l++) {
                cnt += (unsigned)pos[l];
                for (unsigned k = 0; k < cnt; k++)
                    f[bs + l] = (float)((double)f[bs + l] + (double)mt.mod_mass[nums[k]] / (double)scale);
                spec[bs + l] = (uint32_t)(f[bs + l] * (float)scale / (float)(z + 1));
            }
        }
        for (unsigned z = 0; z < maxz; z++) {
            const unsigned ys = z * n1 + maxz * n1;
            unsigned cnt = 0;
            for (int l = (int)n1; l > 0; l--) {
                cnt += (unsigned)pos[l];
                const unsigned o = ys + n1 - (unsigned)l;
                for (unsigned k = 0; k < cnt; k++)
                    f[o] = (float)((double)f[o] + (double)mt.mod_mass[nums[seen - 1 - (int)k]] / (double)scale);
                spec[o] = (uint32_t)(f[o] * (float)scale / (float)(z + 1));
            }
        }
    }
    *filled = true;
    return mass;
}

}  // namespace

struct gx_host_length {
    uint32_t L = 0, maxz = 0, speclen = 0, nbins = 0;
    std::vector<char> seqs;             // kept peptides, npep_kept x L
    std::vector<gx_pep_entry> entries;  // mass-sorted
    std::vector<float> mass;
    std::vector<uint32_t> bA, iA;
};

extern "C" gx_status gx_build_length(const char *seqs, uint32_t npep, uint32_t L, const gx_build_params *bp,
                                     gx_host_length **out)
{
    using namespace gx;
    if (!out || !bp || (!seqs && npep)) return fail(GX_ERR_INVLD_PTR, "gx_build_length: null argument");
    *out = nullptr;
    if (L < 2 || L > (uint32_t)kMaxSeqLen || bp->maxz < 1 || bp->maxz > 6 || bp->scale == 0 ||
        bp->nmods > (uint32_t)kMaxModTypes || bp->max_mass <= bp->min_mass)
        return fail(GX_ERR_INVLD_PARAM, "gx_build_length: bad parameters");
    const int threads = bp->threads > 0 ? bp->threads : omp_get_max_threads();

    ModTable mt;
    for (int &c : mt.cond_of) c = -1;
    mt.limit = (int)bp->mods_per_pep;
    mt.scale = bp->scale;
    std::memset(mt.mod_mass, 0, sizeof(mt.mod_mass));
    for (uint32_t i = 0; i < bp->nmods; i++) {
        for (int j = 0; j < 4 && bp->mods[i].residues[j]; j++)
            mt.cond_of[(unsigned char)bp->mods[i].residues[j]] = (int)i;
        mt.per_type.push_back((int)bp->mods[i].max_per_pep);
        mt.mod_mass[i] = (uint32_t)(bp->mods[i].mass * (double)bp->scale);
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
        const float m = pep_mass(seqs + (size_t)i * L, L);
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
        std::vector<float> f;
        std::vector<uint32_t> spec(speclen);
        uint32_t *c = cnt[t].data();
        for (uint64_t k = k0; k < k1; k++) {
            const gx_pep_entry &e = h->entries[k];
            bool filled = false;
            const float m = entry_spectrum(&h->seqs[(size_t)e.seqid * L], L, e, bp->maxz, (double)bp->min_mass,
                                           (double)bp->max_mass, mt, f, spec.data(), &filled);
            uint32_t *dst = &bins[(size_t)k * speclen];
            if (filled && m >= (double)bp->min_mass && m <= (double)bp->max_mass) {
                for (uint32_t ion = 0; ion < speclen; ion++) {
                    uint32_t b = spec[ion];
                    if ((double)b >= (double)topbin) b = topbin - 1;
                    dst[ion] = b;
                    c[b]++;
                }
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
    d->bA = h->bA.data();
    d->iA = h->iA.data();
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
