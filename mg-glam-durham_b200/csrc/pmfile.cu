// PM snapshot files in the reference's format (WriteDataPM / ReadDataPM,
// PMP2mod_tools.f90:237-487; big-endian, `-convert big_endian`, makefile:6),
// so snapshots move between this library and the Fortran tools.  Host code.
#include "../../include/mgglam.h"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace {

constexpr int64_t kRecord = 1024 * 1024;   // particles per direct-access record
constexpr int64_t kRecordsPerFile = 512;   // Nrecpage
constexpr int kHeaderBytes = 529;

std::mutex g_pm_mu;
std::string g_pm_err;

int fail(int code, const std::string& m) {
    std::lock_guard<std::mutex> lk(g_pm_mu);
    g_pm_err = m;
    return code;
}

template <class T>
void put_be(std::vector<unsigned char>& b, T v) {
    unsigned char raw[sizeof(T)];
    std::memcpy(raw, &v, sizeof(T));
    for (int i = (int)sizeof(T) - 1; i >= 0; --i) b.push_back(raw[i]);
}
template <class T>
T get_be(const unsigned char*& p) {
    unsigned char raw[sizeof(T)];
    for (int i = (int)sizeof(T) - 1; i >= 0; --i) raw[i] = *p++;
    T v;
    std::memcpy(&v, raw, sizeof(T));
    return v;
}

std::string join(const char* dir, const std::string& name) {
    std::string d = dir ? dir : "";
    if (!d.empty() && d.back() != '/') d += '/';
    return d + name;
}
std::string crd_name(int moment) {
    char b[64];
    if (moment < 0) std::snprintf(b, sizeof(b), "PMcrd.DAT");
    else std::snprintf(b, sizeof(b), "PMcrd.%04d.DAT", moment);
    return b;
}
std::string crs_name(int ifile, int moment) {
    char b[64];
    if (moment < 0) std::snprintf(b, sizeof(b), "PMcrs%d.DAT", ifile);
    else std::snprintf(b, sizeof(b), "PMcrs%d.%04d.DAT", ifile, moment);
    return b;
}

std::vector<unsigned char> encode_header(const mgg_pm_header& h) {
    std::vector<unsigned char> b;
    b.reserve(kHeaderBytes);
    for (int i = 0; i < 45; ++i) b.push_back((unsigned char)h.header[i]);
    for (float v : {h.aexpn, h.aexp0, h.amplt, h.astep}) put_be(b, v);
    put_be(b, h.istep);
    for (float v : {h.partw, h.tintg, h.ekin, h.ekin1, h.ekin2, h.au0, h.aeu0}) put_be(b, v);
    for (int32_t v : {h.nrow, h.ngrid, h.nrealization, h.nseed}) put_be(b, v);
    for (float v : {h.om, h.oml, h.hubble}) put_be(b, v);
    put_be(b, h.nparticles);
    for (int i = 0; i < 100; ++i) put_be(b, h.extras[i]);
    return b;
}

void decode_header(const unsigned char* p, mgg_pm_header& h) {
    std::memcpy(h.header, p, 45);
    p += 45;
    h.aexpn = get_be<float>(p); h.aexp0 = get_be<float>(p); h.amplt = get_be<float>(p); h.astep = get_be<float>(p);
    h.istep = get_be<int32_t>(p);
    h.partw = get_be<float>(p); h.tintg = get_be<float>(p); h.ekin = get_be<float>(p); h.ekin1 = get_be<float>(p);
    h.ekin2 = get_be<float>(p); h.au0 = get_be<float>(p); h.aeu0 = get_be<float>(p);
    h.nrow = get_be<int32_t>(p); h.ngrid = get_be<int32_t>(p); h.nrealization = get_be<int32_t>(p);
    h.nseed = get_be<int32_t>(p);
    h.om = get_be<float>(p); h.oml = get_be<float>(p); h.hubble = get_be<float>(p);
    h.nparticles = get_be<int64_t>(p);
    for (int i = 0; i < 100; ++i) h.extras[i] = get_be<float>(p);
}

void swap_floats(const float* src, unsigned char* dst, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        unsigned char raw[4];
        std::memcpy(raw, src + i, 4);
        dst[4 * i] = raw[3]; dst[4 * i + 1] = raw[2]; dst[4 * i + 2] = raw[1]; dst[4 * i + 3] = raw[0];
    }
}
void unswap_floats(const unsigned char* src, float* dst, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        unsigned char raw[4] = {src[4 * i + 3], src[4 * i + 2], src[4 * i + 1], src[4 * i]};
        std::memcpy(dst + i, raw, 4);
    }
}

}  // namespace

extern "C" {

int mgg_pm_write(const char* dir, int32_t moment, const mgg_pm_header* h, const float* x, const float* y,
                 const float* z, const float* vx, const float* vy, const float* vz) {
    if (!h || !x || !y || !z || !vx || !vy || !vz || h->nparticles < 1) return fail(MGG_ERR_ARG, "pm_write: bad argument");
    // PMcrd: one sequential unformatted record
    {
        const std::string name = join(dir, crd_name(moment));
        FILE* f = std::fopen(name.c_str(), "wb");
        if (!f) return fail(MGG_ERR_ARG, "pm_write: cannot open " + name);
        std::vector<unsigned char> rec;
        put_be<int32_t>(rec, kHeaderBytes);
        const std::vector<unsigned char> hb = encode_header(*h);
        rec.insert(rec.end(), hb.begin(), hb.end());
        put_be<int32_t>(rec, kHeaderBytes);
        const bool ok = std::fwrite(rec.data(), 1, rec.size(), f) == rec.size();
        std::fclose(f);
        if (!ok) return fail(MGG_ERR_ARG, "pm_write: short write of " + name);
    }
    // PMcrs: direct-access records of 6 x 1024^2 big-endian floats
    const int64_t np = h->nparticles;
    const int64_t npages = (np - 1) / kRecord + 1;
    std::vector<unsigned char> rec(6 * kRecord * 4);
    std::vector<float> page(kRecord);
    FILE* f = nullptr;
    for (int64_t i = 0; i < npages; ++i) {
        if (i % kRecordsPerFile == 0) {
            if (f) std::fclose(f);
            const std::string name = join(dir, crs_name((int)(i / kRecordsPerFile), moment));
            f = std::fopen(name.c_str(), "wb");
            if (!f) return fail(MGG_ERR_ARG, "pm_write: cannot open " + name);
        }
        const int64_t first = i * kRecord, nin = (i == npages - 1) ? np - first : kRecord;
        const float* src[6] = {x, y, z, vx, vy, vz};
        for (int a = 0; a < 6; ++a) {
            std::memcpy(page.data(), src[a] + first, sizeof(float) * nin);
            if (nin < kRecord) std::memset(page.data() + nin, 0, sizeof(float) * (kRecord - nin));
            swap_floats(page.data(), rec.data() + (size_t)a * kRecord * 4, kRecord);
        }
        if (std::fwrite(rec.data(), 1, rec.size(), f) != rec.size()) {
            std::fclose(f);
            return fail(MGG_ERR_ARG, "pm_write: short write of a particle record");
        }
    }
    if (f) std::fclose(f);
    return MGG_OK;
}

int mgg_pm_read_header(const char* dir, int32_t moment, mgg_pm_header* h) {
    if (!h) return fail(MGG_ERR_ARG, "pm_read_header: null header");
    const std::string name = join(dir, crd_name(moment));
    FILE* f = std::fopen(name.c_str(), "rb");
    if (!f) return fail(MGG_ERR_ARG, "pm_read_header: cannot open " + name);
    unsigned char buf[kHeaderBytes + 8];
    const size_t got = std::fread(buf, 1, sizeof(buf), f);
    std::fclose(f);
    if (got != sizeof(buf)) return fail(MGG_ERR_ARG, "pm_read_header: short file " + name);
    const unsigned char* p = buf;
    const int32_t len = get_be<int32_t>(p);
    if (len != kHeaderBytes) return fail(MGG_ERR_ARG, "pm_read_header: unexpected record length in " + name);
    decode_header(buf + 4, *h);
    return MGG_OK;
}

int mgg_pm_read(const char* dir, int32_t moment, mgg_pm_header* h, float* x, float* y, float* z, float* vx,
                float* vy, float* vz, int64_t capacity) {
    int rc = mgg_pm_read_header(dir, moment, h);
    if (rc != MGG_OK) return rc;
    const int64_t np = h->nparticles;
    if (np < 1 || np > capacity) return fail(MGG_ERR_ARG, "pm_read: particle count exceeds the buffers");
    if (!x || !y || !z || !vx || !vy || !vz) return fail(MGG_ERR_ARG, "pm_read: null buffer");
    const int64_t npages = (np - 1) / kRecord + 1;
    std::vector<unsigned char> rec(6 * kRecord * 4);
    float* dst[6] = {x, y, z, vx, vy, vz};
    std::vector<float> page(kRecord);
    const float xr = (float)(h->ngrid + 1);
    FILE* f = nullptr;
    for (int64_t i = 0; i < npages; ++i) {
        if (i % kRecordsPerFile == 0) {
            if (f) std::fclose(f);
            const std::string name = join(dir, crs_name((int)(i / kRecordsPerFile), moment));
            f = std::fopen(name.c_str(), "rb");
            if (!f) return fail(MGG_ERR_ARG, "pm_read: cannot open " + name);
        }
        if (std::fread(rec.data(), 1, rec.size(), f) != rec.size()) {
            std::fclose(f);
            return fail(MGG_ERR_ARG, "pm_read: short particle record");
        }
        const int64_t first = i * kRecord, nin = (i == npages - 1) ? np - first : kRecord;
        for (int a = 0; a < 6; ++a) {
            unswap_floats(rec.data() + (size_t)a * kRecord * 4, page.data(), nin);
            if (a < 3) {   // boundary guard (PMP2mod_tools.f90:345-347)
                for (int64_t j = 0; j < nin; ++j)
                    if ((int)page[j] == (int)xr) page[j] = page[j] - 1.e-3f;
            }
            std::memcpy(dst[a] + first, page.data(), sizeof(float) * nin);
        }
    }
    if (f) std::fclose(f);
    return MGG_OK;
}

const char* mgg_pm_last_error(void) {
    std::lock_guard<std::mutex> lk(g_pm_mu);
    return g_pm_err.c_str();
}

}  // extern "C"
