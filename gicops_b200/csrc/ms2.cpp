// MS2 text reader: the parsing half of the reference's MS2 -> .pbin conversion
// (source/core/msquery.cpp:137-336, MSQuery::convertAndprepMS2bin), producing the raw
// spectra that gx_pickpeaks_device turns into the query batch.  Same line rules and
// the same C library calls as the reference:
//   - empty lines and lines starting with H or D are skipped;
//   - S starts the next spectrum (the values collected so far belong to the previous
//     one; values before the first S stay with the first spectrum, whose size counts
//     only the lines after its S line, as in the reference);
//   - Z: second field (split on space/tab) = charge, max(1, atoi), default 1; third =
//     precursor M+H, atof as float, default 0.01;
//   - I with second field RTime: third field = retention time, max(0, atof), default 0;
//   - every other line is a peak: split on spaces only (a tab-separated line is one
//     field, its intensity the default), m/z = (int)(atof * scale), intensity =
//     (int)(atof * 100), fields defaulting to "0.01".
// A spectrum without a Z or I line gets the defaults (the reference leaves that slot as
// it was).  The file always yields at least one spectrum, as the reference's does.

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/gicops_b200.h"
#include "gx_internal.h"

struct gx_ms2_file {
    std::vector<uint32_t> seg{0};    // [nspec + 1] each spectrum's collected values
    std::vector<uint32_t> size;      // [nspec] values counted after its S line
    std::vector<int32_t> mz, intn;   // collected values, in file order
    std::vector<float> prec, rtime;
    std::vector<int32_t> charge;
};

namespace {

// double -> int32 as x86's truncating conversion does it (out of range, NaN: INT32_MIN).
int32_t cvt_i32(double v) { return (v >= -2147483648.0 && v < 2147483648.0) ? (int32_t)v : INT32_MIN; }

}  // namespace

extern "C" gx_status gx_ms2_read(const char *path, uint32_t scale, gx_ms2_file **out)
{
    if (!path || !out) return gx::fail(GX_ERR_INVLD_PTR, "gx_ms2_read: null argument");
    *out = nullptr;
    if (scale == 0) return gx::fail(GX_ERR_INVLD_PARAM, "gx_ms2_read: scale must be > 0");
    std::ifstream f(path);
    if (!f.is_open()) return gx::fail(GX_ERR_FILE_NOT_FOUND, std::string("gx_ms2_read: cannot open ") + path);
    auto *h = new gx_ms2_file();
    bool first = true;
    uint32_t specsize = 0;
    auto new_slot = [&]() {
        h->prec.push_back(0.01f);
        h->charge.push_back(1);
        h->rtime.push_back(0.0f);
    };
    auto close_spectrum = [&]() {
        h->size.push_back(specsize);
        h->seg.push_back((uint32_t)h->mz.size());
    };
    new_slot();
    std::string line;
    while (!f.eof()) {
        std::getline(f, line);
        if (line.empty() || line[0] == 'H' || line[0] == 'D') continue;
        std::vector<char> buf(line.begin(), line.end());
        buf.push_back('\0');
        char *save = nullptr;
        if (line[0] == 'S') {
            if (!first) {
                close_spectrum();
                new_slot();
            } else {
                first = false;
            }
            specsize = 0;
        } else if (line[0] == 'Z') {
            char *t = strtok_r(buf.data(), " \t", &save);
            t = strtok_r(nullptr, " \t", &save);
            const int z = std::atoi(t ? t : "1");
            h->charge.back() = z > 1 ? z : 1;
            t = strtok_r(nullptr, " \t", &save);
            h->prec.back() = (float)std::atof(t ? t : "0.01");
        } else if (line[0] == 'I') {
            char *t = strtok_r(buf.data(), " \t", &save);
            t = strtok_r(nullptr, " \t", &save);
            if (t && std::strcmp(t, "RTime") == 0) {
                t = strtok_r(nullptr, " \t", &save);
                const double r = std::atof(t ? t : "0.00");
                h->rtime.back() = (float)(r > 0.0 ? r : 0.0);
            }
        } else {
            char *m = strtok_r(buf.data(), " ", &save);
            char *i = strtok_r(nullptr, " ", &save);
            h->mz.push_back(cvt_i32(std::atof(m ? m : "0.01") * (double)scale));
            h->intn.push_back(cvt_i32(std::atof(i ? i : "0.01") * 100.0));
            specsize++;
        }
    }
    close_spectrum();
    if (h->mz.size() >= (1ull << 32)) {
        delete h;
        return gx::fail(GX_ERR_INVLD_SIZE, "gx_ms2_read: 2^32 or more peaks");
    }
    *out = h;
    return GX_SUCCESS;
}

extern "C" gx_status gx_ms2_desc(const gx_ms2_file *h, gx_ms2_raw *d)
{
    if (!h || !d) return gx::fail(GX_ERR_INVLD_PTR, "gx_ms2_desc: null argument");
    d->nspec = (uint32_t)h->size.size();
    d->nvalues = (uint32_t)h->mz.size();
    d->seg = h->seg.data();
    d->size = h->size.data();
    d->mz = h->mz.data();
    d->intn = h->intn.data();
    d->prec = h->prec.data();
    d->charge = h->charge.data();
    d->rtime = h->rtime.data();
    return GX_SUCCESS;
}

extern "C" void gx_ms2_free(gx_ms2_file *h) { delete h; }
