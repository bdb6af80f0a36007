// Fragment-ion arithmetic of the index build, shared by the host builder (g++) and the
// device builder (nvcc), so that both produce the same bins from the same float and
// double operations in the same order (both are compiled without FMA contraction).
// Paths relative to the reference project:
//   residue masses        cmake/Templates/aamasses.hpp.in:25-80 (double literals narrowed
//                         to float, as the reference's constexpr float tables are)
//   peptide mass          source/core/utils.cpp:240-252
//   variant mass          source/core/utils.cpp:306-331 (only the first modification's
//                         mass is added: the loop's shift count is the mask itself)
//   fragment ions         source/core/utils.cpp:161-226 (unmodified), 347-474 (variants)
//   bins                  source/core/dslim.cpp:231-402 (clamped to the last bin)
#pragma once

#include <stdint.h>

#include "../../include/gicops_b200.h"

#ifdef __CUDACC__
#define GX_HD __host__ __device__ __forceinline__
#else
#define GX_HD inline
#endif

namespace gx {
namespace ions {

constexpr int kMaxSeqLen = 60;
constexpr int kMaxModTypes = 15;
constexpr double kNAA = -20000.0;
constexpr float kH2O = 18.015f;
constexpr float kProton = 1.00727647f;

// Initialisers of the residue tables (A..Z); kNAA for letters that are not residues.
#define GX_AA_MASS_INIT                                                                                             \
    {(float)71.03712, (float)-20000.0, (float)103.00919, (float)115.030, (float)129.0426, (float)147.068,          \
     (float)57.02146, (float)137.060, (float)113.084, (float)-20000.0, (float)128.094, (float)113.084,             \
     (float)131.0405, (float)114.043, (float)-20000.0, (float)97.0527, (float)128.05858, (float)156.1012,          \
     (float)87.032, (float)101.0476, (float)-20000.0, (float)99.06841, (float)186.0793, (float)-20000.0,           \
     (float)163.0633, (float)-20000.0}
#define GX_STAT_MOD_INIT \
    {0, 0, (float)57.021464, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}

// Residue tables and modification masses, held where the caller's code reads them
// (host memory, or shared memory in a kernel).
struct IonTables {
    float aa[26];                     // residue masses
    float stat[26];                   // fixed modifications (carbamidomethyl C)
    uint32_t mod_mass[kMaxModTypes];  // variable modifications, (uint)(mass * scale)
    uint32_t scale;                   // bins per Da
};

GX_HD int aa_index(char c) { return c - 'A'; }

GX_HD float aa_z(const IonTables &t, char c, unsigned z)
{
    return (t.aa[aa_index(c)] + t.stat[aa_index(c)]) + (kProton * (float)z);
}

GX_HD float pep_mass(const IonTables &t, const char *s, unsigned L)
{
    float m = kH2O;
    for (unsigned l = 0; l < L; l++) m += t.aa[aa_index(s[l])] + t.stat[aa_index(s[l])];
    return m;
}

// The reference's loop shifts by the mask (0xF0), which x86 reduces mod 32 to 16, so its
// second pass always reads 0: exactly one modification contributes.
GX_HD float mod_mass_first_only(const IonTables &t, const char *s, unsigned L, uint32_t modnum)
{
    float m = kH2O;
    for (unsigned l = 0; l < L; l++) {
        m += t.aa[aa_index(s[l])];
        m += t.stat[aa_index(s[l])];
    }
    const uint32_t first = modnum & 0x0Fu;
    if (first != 0) m += ((float)t.mod_mass[first - 1]) / (float)t.scale;
    return m;
}

// Whether an entry's ions are binned (else all of them go to bin 0): its mass is positive
// (peptide) or inside (minmass, maxmass) with a site set (variant), and inside
// [minmass, maxmass].
GX_HD bool entry_binned(const IonTables &t, const char *seq, unsigned L, uint64_t sites, uint32_t modnum,
                        double minmass, double maxmass)
{
    float mass;
    if (modnum == 0) {
        mass = pep_mass(t, seq, L);
        if (!(mass > 0)) return false;
    } else {
        if (sites == 0) return false;
        mass = mod_mass_first_only(t, seq, L, modnum);
        if (!(mass > minmass && mass < maxmass)) return false;
    }
    return mass >= minmass && mass <= maxmass;
}

// Modification types (0-based) of a variant's modified sites, from its modnum nibbles
// (type + 1 per site, first site in the lowest nibble); returns the number of sites.
GX_HD int mod_types(uint32_t modnum, int *nums)
{
    int seen = 0;
    uint32_t mask = modnum;
    for (int i = 0; i < kMaxModTypes; i++) {
        nums[i] = (int)(mask & 0x0Fu) - 1;
        mask /= 16;
        if (nums[i] != -1) seen++;
    }
    return seen;
}

// Bins of one ion series of an entry that is binned: charge z + 1 (z = 0..maxz-1), b
// ions (y = false, positions l = 0..L-2 from the N-terminus) or y ions (from the
// C-terminus), written to out[0..L-2]; bins at or above topbin are clamped to topbin - 1.
// Ion l of a variant adds, in double, the mass of every modified site it covers
// (residues 0..l for b ions, taken from the first site on; L-1..L-1-l for y ions, taken
// from the last site back) to the unmodified prefix sum, then rounds to float.
GX_HD void ion_series(const IonTables &t, const char *seq, unsigned L, uint64_t sites, uint32_t modnum, unsigned z,
                      bool y, uint32_t topbin, uint32_t *out)
{
    const unsigned n1 = L - 1;
    const float zs = (float)(z + 1);
    const float sc = (float)t.scale;
    int nums[kMaxModTypes];
    const int seen = modnum != 0 ? mod_types(modnum, nums) : 0;
    float run = y ? aa_z(t, seq[L - 1], z + 1) + kH2O : aa_z(t, seq[0], z + 1);
    unsigned cnt = 0;
    for (unsigned l = 0; l < n1; l++) {
        if (l > 0) run = run + aa_z(t, y ? seq[L - 1 - l] : seq[l], 0);
        float f = run;
        if (modnum != 0) {
            const unsigned site = y ? n1 - l : l;
            cnt += (unsigned)((sites >> site) & 1u);
            for (unsigned k = 0; k < cnt; k++) {
                const int idx = y ? seen - 1 - (int)k : (int)k;
                const int m = (idx >= 0 && idx < kMaxModTypes) ? nums[idx] : -1;
                const double add = m >= 0 ? (double)t.mod_mass[m] / (double)t.scale : 0.0;
                f = (float)((double)f + add);
            }
        }
        uint32_t b = (uint32_t)((f * sc) / zs);
        if ((double)b >= (double)topbin) b = topbin - 1;
        out[l] = b;
    }
}

}  // namespace ions

// Tables of a build: the residue masses, and each modification's mass as the reference
// stores it, (uint)(mass * scale) (source/apps/argp/argp.hpp:359).
inline ions::IonTables ion_tables(const gx_build_params *bp)
{
    ions::IonTables t = {GX_AA_MASS_INIT, GX_STAT_MOD_INIT, {0}, bp->scale};
    for (uint32_t i = 0; i < bp->nmods && i < (uint32_t)ions::kMaxModTypes; i++)
        t.mod_mass[i] = (uint32_t)(bp->mods[i].mass * (double)bp->scale);
    return t;
}

}  // namespace gx
