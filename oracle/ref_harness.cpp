// Test infrastructure only (oracle side).  Drives the reference's own CPU query
// path, compiled unchanged from its sources by oracle/Makefile, so that tests and
// the reference arm of bench.py can compare against it.  It is never linked into
// the product.
//
// What it does, in the order source/apps/gicops/gicops.cpp:96-271 does it:
//   UTILS_InitializeModInfo -> MODS_Initialize -> per length L:
//   LBE_CountPeps -> LBE_CreatePartitions -> LBE_Initialize -> LBE_Distribute ->
//   DSLIM_Construct; then DSLIM_DeallocateSpecArr, DSLIM_InitializeScorecard, and
//   DSLIM_QuerySpectrum (source/core/dslim_query.cpp:749) per batch of QCHUNK
//   spectra read from a .pbin file (layout of source/core/msquery.cpp:425-462).
// DFile_PrintScore (source/core/dslim_fileout.cpp:112) is replaced here: it records
// the exact float hyperscore, psid, idxoffset, shared ions and double e-value of
// every reported PSM instead of formatting a TSV row.
//
// Usage:
//   ref_harness --db DIR --minlen 6 --maxlen 46 --maxz 1 --dM 10 --dF 5
//               [--mods M:15.9949:2 ...] [--nmods 2] [--threads N] [--topmatches 5]
//               [--expect-max 1e300] [--queries Q.pbin] [--first N] [--repeat R]
//               [--out RES.bin] [--dump-index IDX.bin] [--qdm DM.f64]
//               [--min-cpsm 4] [--min-shp 4] [--entries-only] [--batch Q.pbin:DM ...]
//   ref_harness --ms2-to-pbin FILE.ms2     (the reference's MS2 conversion: FILE.ms2.pbin)
// --batch (repeatable) searches several query files, each at its own global tolerance DM
// (Da), against one index build; each repeat runs them all and is timed as their sum.
// --entries-only stops after the index entries (LBE_* steps, no fragment-ion index) and,
// with --dump-index, writes them alone (magic GXREFEN1: no bA / iA arrays).
// --qdm gives one precursor tolerance (Da, float64) per spectrum: each spectrum is then
// searched alone with params.dM set to its value (the reference reads params.dM at
// call time in DSLIM_BinarySearch, source/core/dslim_query.cpp:1102-1106).
// Prints one JSON line with timings last.

#include <omp.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "common.hpp"
#include "config.hpp"
#include "dslim.h"
#include "dslim_fileout.h"
#include "msquery.hpp"
#include "expeRT.h"
#include "lbe.h"
#include "mods.h"
#include "scheduler.h"
#include "slm_dsts.h"
#include "utils.h"

gParams params;
std::vector<string_t> queryfiles;

extern Scheduler *SchedHandle;
extern expeRT *ePtrs;
extern BYICount *Score;

namespace {

struct Capture {
    int32_t reported;
    int32_t psid;
    uint16_t idxoffset;
    uint16_t sharedions;
    uint16_t totalions;
    uint16_t pad0;
    float hyperscore;
    uint32_t npsms;
    double e_x;
};
static_assert(sizeof(Capture) == 32, "capture record is 32 bytes");

std::vector<Capture> g_capture;

}  // namespace

status_t DFile_InitFiles() { return SLM_SUCCESS; }
status_t DFile_DeinitFiles() { return SLM_SUCCESS; }
status_t DFile_PrintPartials(uint_t, Results *) { return SLM_SUCCESS; }

status_t DFile_PrintScore(Index *, uint_t specid, float_t, hCell *psm, double_t e_x, uint_t npsms)
{
    if (specid < g_capture.size()) {
        Capture &c = g_capture[specid];
        c.reported = 1;
        c.psid = psm->psid;
        c.idxoffset = psm->idxoffset;
        c.sharedions = psm->sharedions;
        c.totalions = psm->totalions;
        c.hyperscore = psm->hyperscore;
        c.npsms = npsms;
        c.e_x = e_x;
    }
    return SLM_SUCCESS;
}

static double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Spec {
    float prec;
    int z;
    float rt;
    std::vector<int> mz, in;
};

static bool read_pbin(const std::string &path, std::vector<Spec> &out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    while (true) {
        Spec s;
        int len = 0;
        if (!f.read((char *)&s.prec, 4)) break;
        f.read((char *)&s.z, 4);
        f.read((char *)&s.rt, 4);
        f.read((char *)&len, 4);
        if (!f || len < 0) return false;
        s.mz.resize(len);
        s.in.resize(len);
        f.read((char *)s.mz.data(), 4 * (size_t)len);
        f.read((char *)s.in.data(), 4 * (size_t)len);
        if (!f) return false;
        out.push_back(std::move(s));
    }
    return true;
}

// The reference's MS2 -> .pbin converter (source/core/msquery.cpp:137-336: parsing, peak
// picking and intensity normalisation of msquery.cpp:338-423) is a protected static member.
struct Ms2Converter : MSQuery {
    static std::array<int, 2> run(std::string *path) { return convertAndprepMS2bin(path); }
};

int main(int argc, char **argv)
{
    std::string db, qpath, outpath, dumppath, qdmpath, ms2path;
    std::vector<std::string> mods;
    std::vector<std::pair<std::string, double>> batches;   // --batch PATH:DM
    int minlen = 6, maxlen = 46, maxz = 1, nmods = 0, threads = omp_get_max_threads();
    int topmatches = 5, first = -1, repeat = 1, min_cpsm = 4, min_shp = 4;
    double dM = 10.0, expect_max = 1e300;
    unsigned dF = 5;
    bool entries_only = false;

    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto nxt = [&]() -> std::string {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "--db") db = nxt();
        else if (a == "--minlen") minlen = std::atoi(nxt().c_str());
        else if (a == "--maxlen") maxlen = std::atoi(nxt().c_str());
        else if (a == "--maxz") maxz = std::atoi(nxt().c_str());
        else if (a == "--dM") dM = std::atof(nxt().c_str());
        else if (a == "--dF") dF = (unsigned)std::atoi(nxt().c_str());
        else if (a == "--mods") mods.push_back(nxt());
        else if (a == "--nmods") nmods = std::atoi(nxt().c_str());
        else if (a == "--threads") threads = std::atoi(nxt().c_str());
        else if (a == "--topmatches") topmatches = std::atoi(nxt().c_str());
        else if (a == "--expect-max") expect_max = std::atof(nxt().c_str());
        else if (a == "--queries") qpath = nxt();
        else if (a == "--first") first = std::atoi(nxt().c_str());
        else if (a == "--repeat") repeat = std::atoi(nxt().c_str());
        else if (a == "--out") outpath = nxt();
        else if (a == "--dump-index") dumppath = nxt();
        else if (a == "--qdm") qdmpath = nxt();
        else if (a == "--min-cpsm") min_cpsm = std::atoi(nxt().c_str());
        else if (a == "--min-shp") min_shp = std::atoi(nxt().c_str());
        else if (a == "--ms2-to-pbin") ms2path = nxt();
        else if (a == "--entries-only") entries_only = true;
        else if (a == "--batch") {
            const std::string v = nxt();
            const size_t c = v.rfind(':');
            if (c == std::string::npos) { std::fprintf(stderr, "--batch wants PATH:DM\n"); return 2; }
            batches.emplace_back(v.substr(0, c), std::atof(v.c_str() + c + 1));
        }
        else { std::fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }
    if (!ms2path.empty()) {
        // writes <ms2path>.pbin with the reference's default scale and intensity parameters
        params.scale = 100;
        params.base_int = 1000 * YAXISMULTIPLIER;
        params.min_int = (int)(params.base_int * 0.01 + 0.5);
        const std::array<int, 2> r = Ms2Converter::run(&ms2path);
        std::printf("{\"spectra\": %d, \"largest\": %d}\n", r[0], r[1]);
        return 0;
    }
    if (db.empty()) { std::fprintf(stderr, "--db is required\n"); return 2; }

    // Parameters as source/apps/argp/argp.hpp:215-386 would set them.
    params.threads = threads;
    params.maxprepthds = 1;
    params.gputhreads = 0;
    params.min_len = minlen;
    params.max_len = maxlen;
    params.maxz = maxz;
    params.topmatches = topmatches;
    params.scale = 100;
    params.res = 0.01;
    params.dF = dF;
    params.dM = dM;
    params.min_mass = 500;
    params.max_mass = 5000;
    params.min_shp = min_shp;
    params.min_cpsm = min_cpsm;
    params.expect_max = expect_max;
    params.base_int = 1000 * YAXISMULTIPLIER;
    params.min_int = (int)(params.base_int * 0.01 + 0.5);
    params.spadmem = 0xF0000000u;  // large: one chunk per length (nChunks == 1)
    params.nodes = 1;
    params.myid = 0;
    params.useGPU = false;
    params.gpuindex = false;
    params.policy = DistPolicy_t::cyclic;
    params.vModInfo.vmods_per_pep = nmods;
    params.vModInfo.num_vars = mods.size();
    if (!mods.empty()) {
        params.modconditions = std::to_string(nmods);
        for (size_t md = 0; md < mods.size(); md++) {
            std::string m = mods[md];
            size_t c1 = m.find(':'), c2 = m.rfind(':');
            std::string aa = m.substr(0, c1), mass = m.substr(c1 + 1, c2 - c1 - 1), num = m.substr(c2 + 1);
            params.modconditions += " " + aa;
            std::strncpy((char *)params.vModInfo.vmods[md].residues, aa.c_str(), std::min<size_t>(4, aa.size()));
            params.vModInfo.vmods[md].modMass = (uint_t)(std::atof(mass.c_str()) * params.scale);
            params.modconditions += " " + num;
            params.vModInfo.vmods[md].aa_per_peptide = std::atoi(num.c_str());
        }
    } else {
        params.vModInfo.num_vars = 0;
        params.modconditions = "0";
    }
    queryfiles.push_back("synthetic.pbin");

    status_t st = UTILS_InitializeModInfo(&params.vModInfo);
    if (st == SLM_SUCCESS) st = MODS_Initialize();

    const int nlen = maxlen - minlen + 1;
    Index *index = new Index[nlen];
    double t0 = now_s();
    for (int L = minlen; L <= maxlen && st == SLM_SUCCESS; L++) {
        std::string file = db + "/" + std::to_string(L) + ".peps";
        Index *ix = index + (L - minlen);
        ix->pepIndex.peplen = L;
        st = LBE_CountPeps(file, ix, L);
        if (st == SLM_SUCCESS) st = LBE_CreatePartitions(ix);
        if (st == SLM_SUCCESS) st = LBE_Initialize(ix);
        if (st == SLM_SUCCESS) st = LBE_Distribute(ix);
        if (st == SLM_SUCCESS && ix->nChunks != 1) {
            std::fprintf(stderr, "length %d split into %u chunks\n", L, ix->nChunks);
            st = ERR_INVLD_SIZE;
        }
        if (st == SLM_SUCCESS && !entries_only) st = DSLIM_Construct(ix);
    }
    if (st == SLM_SUCCESS && !entries_only) st = DSLIM_DeallocateSpecArr();
    if (st == SLM_SUCCESS && !entries_only) st = DSLIM_InitializeScorecard(index, nlen);
    double t1 = now_s();
    if (st != SLM_SUCCESS) { std::fprintf(stderr, "index build failed: %d\n", st); return 1; }

    if (!dumppath.empty()) {
        FILE *f = std::fopen(dumppath.c_str(), "wb");
        if (!f) { std::perror("dump"); return 1; }
        const uint32_t nb = (uint32_t)(params.max_mass * params.scale) + 1;
        std::fwrite(entries_only ? "GXREFEN1" : "GXREFIX1", 1, 8, f);
        int32_t hdr[4] = {nlen, minlen, maxz, (int32_t)nb};
        std::fwrite(hdr, 4, 4, f);
        for (int i = 0; i < nlen; i++) {
            Index *ix = index + i;
            const uint32_t L = ix->pepIndex.peplen, N = ix->lcltotCnt, npep = ix->lclpepCnt;
            const uint32_t speclen = (L - 1) * maxz * iSERIES;
            uint32_t h[4] = {L, N, npep, speclen};
            std::fwrite(h, 4, 4, f);
            std::fwrite(ix->pepIndex.seqs, 1, (size_t)npep * L, f);
            for (uint32_t k = 0; k < N; k++) std::fwrite(&ix->pepEntries[k].Mass, 4, 1, f);
            for (uint32_t k = 0; k < N; k++) std::fwrite(&ix->pepEntries[k].seqID, 4, 1, f);
            for (uint32_t k = 0; k < N; k++) std::fwrite(&ix->pepEntries[k].sites.sites, 8, 1, f);
            for (uint32_t k = 0; k < N; k++) std::fwrite(&ix->pepEntries[k].sites.modNum, 4, 1, f);
            if (entries_only) continue;
            std::fwrite(ix->ionIndex[0].bA, 4, nb, f);
            std::fwrite(ix->ionIndex[0].iA, 4, (size_t)N * speclen, f);
        }
        std::fclose(f);
    }

    double tq = 0.0;
    std::vector<double> t_each;
    size_t nspec = 0;
    if (!qpath.empty()) batches.insert(batches.begin(), std::make_pair(qpath, dM));
    if (!batches.empty() && !entries_only) {
        // every batch read up front; with a single batch, --first and --qdm apply to it
        std::vector<std::vector<Spec>> all(batches.size());
        for (size_t bi = 0; bi < batches.size(); bi++)
            if (!read_pbin(batches[bi].first, all[bi])) {
                std::fprintf(stderr, "bad pbin %s\n", batches[bi].first.c_str());
                return 1;
            }
        if (first >= 0 && all.size() == 1 && (size_t)first < all[0].size()) all[0].resize(first);
        for (auto &v : all) nspec += v.size();
        g_capture.assign(nspec, Capture{});

        SchedHandle = new Scheduler(0);
        ePtrs = new expeRT[params.threads];

        Queries<int> q;
        const int chunk = QCHUNK;
        size_t maxpk = 0;
        for (auto &v : all)
            for (auto &sp : v) maxpk = std::max(maxpk, sp.mz.size());
        q.idx = new uint_t[chunk + 1];
        q.precurse = new float_t[chunk];
        q.charges = new int_t[chunk];
        q.rtimes = new float_t[chunk];
        q.moz = new int[(size_t)chunk * std::max<size_t>(maxpk, 1)];
        q.intensity = new int[(size_t)chunk * std::max<size_t>(maxpk, 1)];

        std::vector<double> qdm;
        if (!qdmpath.empty()) {
            if (all.size() != 1) { std::fprintf(stderr, "--qdm needs a single batch\n"); return 1; }
            qdm.resize(nspec);
            FILE *f = std::fopen(qdmpath.c_str(), "rb");
            if (!f || std::fread(qdm.data(), 8, nspec, f) != nspec) { std::fprintf(stderr, "bad --qdm\n"); return 1; }
            std::fclose(f);
        }
        const size_t step = qdm.empty() ? (size_t)chunk : 1;
        for (int r = 0; r < repeat; r++) {
            const double tq0 = tq;
            size_t base = 0;   // spectrum id of the batch's first spectrum (capture order)
            for (size_t bi = 0; bi < all.size(); bi++) {
                const std::vector<Spec> &specs = all[bi];
                params.dM = batches[bi].second;
                for (size_t b0 = 0; b0 < specs.size(); b0 += step) {
                    const size_t b1 = std::min(specs.size(), b0 + step);
                    if (!qdm.empty()) params.dM = qdm[b0];
                    size_t ind = 0;
                    q.idx[0] = 0;
                    for (size_t s = b0; s < b1; s++) {
                        const Spec &sp = specs[s];
                        q.precurse[s - b0] = sp.prec;
                        q.charges[s - b0] = sp.z;
                        q.rtimes[s - b0] = sp.rt;
                        std::memcpy(q.moz + ind, sp.mz.data(), 4 * sp.mz.size());
                        std::memcpy(q.intensity + ind, sp.in.data(), 4 * sp.in.size());
                        ind += sp.mz.size();
                        q.idx[s - b0 + 1] = (uint_t)ind;
                    }
                    q.numPeaks = (int)ind;
                    q.numSpecs = (int)(b1 - b0);
                    q.batchNum = (int)(b0 / chunk);
                    q.fileNum = 0;
                    double a = now_s();
                    st = DSLIM_QuerySpectrum(&q, index, (uint_t)nlen, (int)(base + b0));
                    tq += now_s() - a;
                    if (st != SLM_SUCCESS) { std::fprintf(stderr, "query failed: %d\n", st); return 1; }
                }
                base += specs.size();
            }
            t_each.push_back(tq - tq0);
        }
        if (!outpath.empty()) {
            FILE *f = std::fopen(outpath.c_str(), "wb");
            if (!f) { std::perror("out"); return 1; }
            std::fwrite(g_capture.data(), sizeof(Capture), g_capture.size(), f);
            std::fclose(f);
        }
    }

    std::string each = "[";
    for (size_t i = 0; i < t_each.size(); i++) each += (i ? ", " : "") + std::to_string(t_each[i]);
    each += "]";
    std::printf("\n{\"index_s\": %.6f, \"query_s\": %.6f, \"query_s_each\": %s, \"nspec\": %zu, "
                "\"repeat\": %d, \"threads\": %d}\n",
                t1 - t0, tq, each.c_str(), nspec, repeat, params.threads);
    return 0;
}
