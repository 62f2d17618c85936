// ncdf.cpp -- netCDF-3 classic files of a 3-component field, without libnetcdf.
//
// The reference keeps its velocity fields (u_result_*.nc, restart and
// perturbation inputs) in netCDF classic files written by
// save_field_R3toR3_ncdf (data_ops.f90:362-487) and read by
// read_field_R3toR3_ncdf (data_ops.f90:1198-1397).  For N >= 16 it writes
// with parallel_data set (initialize.f90:196-201): dimensions "x", "y" and an
// unlimited "z", and three NC_DOUBLE record variables (one z plane per
// record, x fastest), no attributes, created with NF90_CLOBBER (the classic
// CDF-1 format).  This file restates the published classic format (header:
// magic, record count, dimension, attribute and variable lists in big-endian
// 32-bit words, names padded to four bytes; data: fixed-size variables, then
// the records, each the record variables' slabs in definition order) for
// exactly that use: the writer produces that layout, the reader accepts it,
// the fixed-size layout of the serial path (data_ops.f90:455-487) and the
// 64-bit-offset variant (CDF-2), and skips attributes of any type.
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "maxlq.h"

namespace {

constexpr uint32_t TAG_DIMENSION = 0x0A, TAG_VARIABLE = 0x0B, TAG_ATTRIBUTE = 0x0C;
constexpr uint32_t T_BYTE = 1, T_CHAR = 2, T_SHORT = 3, T_INT = 4, T_FLOAT = 5, T_DOUBLE = 6;

uint32_t type_size(uint32_t t) {
    switch (t) {
        case T_BYTE:
        case T_CHAR: return 1;
        case T_SHORT: return 2;
        case T_INT:
        case T_FLOAT: return 4;
        case T_DOUBLE: return 8;
        default: return 0;
    }
}
uint64_t pad4(uint64_t v) { return (v + 3) & ~uint64_t(3); }

struct Var {
    std::string name;
    std::vector<uint32_t> dims;
    uint32_t type = 0;
    uint64_t vsize = 0, begin = 0;
};
struct Header {
    int version = 0;
    uint64_t numrecs = 0;
    std::vector<std::string> dim_names;
    std::vector<uint64_t> dim_len;  // 0 for the record dimension
    int recdim = -1;
    std::vector<Var> vars;
    uint64_t recsize = 0;  // bytes of one record (all record variables)
};

// big-endian encoding
struct Out {
    std::vector<unsigned char> b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void name(const std::string& s) {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        while (b.size() % 4) b.push_back(0);
    }
};

struct In {
    FILE* f;
    bool ok = true;
    uint32_t u32() {
        unsigned char c[4];
        if (std::fread(c, 1, 4, f) != 4) ok = false;
        return ((uint32_t)c[0] << 24) | ((uint32_t)c[1] << 16) | ((uint32_t)c[2] << 8) | c[3];
    }
    uint64_t u64() {
        const uint64_t hi = u32();
        return (hi << 32) | u32();
    }
    std::string name() {
        const uint32_t n = u32();
        if (!ok || n > 4096) {
            ok = false;
            return {};
        }
        std::string s(pad4(n), '\0');
        if (std::fread(&s[0], 1, s.size(), f) != s.size()) ok = false;
        s.resize(n);
        return s;
    }
    void skip(uint64_t n) {
        if (std::fseek(f, (long)n, SEEK_CUR) != 0) ok = false;
    }
};

bool read_att_list(In& in) {
    const uint32_t tag = in.u32(), n = in.u32();
    if (tag == 0 && n == 0) return in.ok;
    if (tag != TAG_ATTRIBUTE) return false;
    for (uint32_t i = 0; i < n && in.ok; ++i) {
        in.name();
        const uint32_t t = in.u32(), cnt = in.u32();
        const uint32_t s = type_size(t);
        if (!s) return false;
        in.skip(pad4((uint64_t)cnt * s));
    }
    return in.ok;
}

bool read_header(FILE* f, Header& h) {
    In in{f};
    unsigned char magic[4];
    if (std::fread(magic, 1, 4, f) != 4 || magic[0] != 'C' || magic[1] != 'D' || magic[2] != 'F' ||
        (magic[3] != 1 && magic[3] != 2))
        return false;
    h.version = magic[3];
    h.numrecs = in.u32();
    {
        const uint32_t tag = in.u32(), n = in.u32();
        if (!(tag == 0 && n == 0)) {
            if (tag != TAG_DIMENSION) return false;
            for (uint32_t i = 0; i < n && in.ok; ++i) {
                h.dim_names.push_back(in.name());
                h.dim_len.push_back(in.u32());
                if (h.dim_len.back() == 0) h.recdim = (int)i;
            }
        }
    }
    if (!read_att_list(in)) return false;
    {
        const uint32_t tag = in.u32(), n = in.u32();
        if (!(tag == 0 && n == 0)) {
            if (tag != TAG_VARIABLE) return false;
            for (uint32_t i = 0; i < n && in.ok; ++i) {
                Var v;
                v.name = in.name();
                const uint32_t nd = in.u32();
                if (nd > 64) return false;
                for (uint32_t k = 0; k < nd; ++k) {
                    v.dims.push_back(in.u32());
                    if (v.dims.back() >= h.dim_len.size()) return false;
                }
                if (!read_att_list(in)) return false;
                v.type = in.u32();
                v.vsize = in.u32();
                v.begin = h.version == 2 ? in.u64() : in.u32();
                h.vars.push_back(v);
            }
        }
    }
    int nrec = 0;
    for (const Var& v : h.vars)
        if (!v.dims.empty() && (int)v.dims[0] == h.recdim) {
            h.recsize += v.vsize;
            ++nrec;
        }
    // a single record variable's records are not padded
    if (nrec == 1)
        for (const Var& v : h.vars)
            if (!v.dims.empty() && (int)v.dims[0] == h.recdim) {
                uint64_t e = type_size(v.type);
                for (size_t k = 1; k < v.dims.size(); ++k) e *= h.dim_len[v.dims[k]];
                h.recsize = e;
            }
    return in.ok;
}

// big-endian doubles <-> host
void put_be_doubles(const double* src, size_t n, unsigned char* dst) {
    for (size_t i = 0; i < n; ++i) {
        uint64_t v;
        std::memcpy(&v, src + i, 8);
        for (int s = 0; s < 8; ++s) dst[8 * i + s] = (unsigned char)(v >> (56 - 8 * s));
    }
}
void get_be_doubles(const unsigned char* src, size_t n, double* dst) {
    for (size_t i = 0; i < n; ++i) {
        uint64_t v = 0;
        for (int s = 0; s < 8; ++s) v = (v << 8) | src[8 * i + s];
        std::memcpy(dst + i, &v, 8);
    }
}

struct FileGuard {
    FILE* f;
    ~FileGuard() {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

int mlq_ncdf_write_field(const char* path, int n1, int n2, int n3, const double* u, const char* name1,
                         const char* name2, const char* name3) {
    if (!path || !u || !name1 || !name2 || !name3 || n1 < 1 || n2 < 1 || n3 < 1) return MLQ_ERR_BADARG;
    const uint64_t slab = (uint64_t)n1 * n2 * 8;
    if (slab >= 0xFFFFFFFCull) return MLQ_ERR_BADARG;  // the 32-bit vsize of the classic format
    const char* names[3] = {name1, name2, name3};
    Out h;
    const unsigned char magic[4] = {'C', 'D', 'F', 1};
    h.b.insert(h.b.end(), magic, magic + 4);
    h.u32((uint32_t)n3);  // numrecs
    h.u32(TAG_DIMENSION);
    h.u32(3);
    h.name("x");
    h.u32((uint32_t)n1);
    h.name("y");
    h.u32((uint32_t)n2);
    h.name("z");
    h.u32(0);  // unlimited
    h.u32(0);  // no global attributes
    h.u32(0);
    h.u32(TAG_VARIABLE);
    h.u32(3);
    std::vector<size_t> begin_at(3);
    for (int k = 0; k < 3; ++k) {
        h.name(names[k]);
        h.u32(3);
        h.u32(2);  // z (record), y, x: x varies fastest
        h.u32(1);
        h.u32(0);
        h.u32(0);  // no attributes
        h.u32(0);
        h.u32(T_DOUBLE);
        h.u32((uint32_t)slab);
        begin_at[k] = h.b.size();
        h.u32(0);  // begin, filled in below
    }
    const uint64_t hdr = h.b.size();  // a multiple of 4: the records start here
    for (int k = 0; k < 3; ++k) {
        const uint64_t b = hdr + (uint64_t)k * slab;
        if (b > 0xFFFFFFFFull) return MLQ_ERR_BADARG;
        for (int s = 0; s < 4; ++s) h.b[begin_at[k] + s] = (unsigned char)(b >> (24 - 8 * s));
    }
    FileGuard g{std::fopen(path, "wb")};
    if (!g.f) return MLQ_ERR_IO;
    if (std::fwrite(h.b.data(), 1, h.b.size(), g.f) != h.b.size()) return MLQ_ERR_IO;
    const size_t nxy = (size_t)n1 * n2;
    std::vector<unsigned char> buf(slab);
    for (int z = 0; z < n3; ++z)
        for (int k = 0; k < 3; ++k) {
            put_be_doubles(u + ((size_t)k * n3 + z) * nxy, nxy, buf.data());
            if (std::fwrite(buf.data(), 1, buf.size(), g.f) != buf.size()) return MLQ_ERR_IO;
        }
    if (std::fclose(g.f) != 0) {
        g.f = nullptr;
        return MLQ_ERR_IO;
    }
    g.f = nullptr;
    return MLQ_OK;
}

int mlq_ncdf_read_dims(const char* path, int dims[3]) {
    if (!path || !dims) return MLQ_ERR_BADARG;
    FileGuard g{std::fopen(path, "rb")};
    if (!g.f) return MLQ_ERR_IO;
    Header h;
    if (!read_header(g.f, h)) return MLQ_ERR_IO;
    const char* want[3] = {"x", "y", "z"};
    for (int k = 0; k < 3; ++k) {
        dims[k] = -1;
        for (size_t i = 0; i < h.dim_names.size(); ++i)
            if (h.dim_names[i] == want[k]) dims[k] = (int)((int)i == h.recdim ? h.numrecs : h.dim_len[i]);
        if (dims[k] < 0) return MLQ_ERR_BADARG;
    }
    return MLQ_OK;
}

int mlq_ncdf_read_field(const char* path, int n1, int n2, int n3, double* u, const char* name1, const char* name2,
                        const char* name3) {
    if (!path || !u || !name1 || !name2 || !name3 || n1 < 1 || n2 < 1 || n3 < 1) return MLQ_ERR_BADARG;
    FileGuard g{std::fopen(path, "rb")};
    if (!g.f) return MLQ_ERR_IO;
    Header h;
    if (!read_header(g.f, h)) return MLQ_ERR_IO;
    const char* names[3] = {name1, name2, name3};
    const size_t nxy = (size_t)n1 * n2;
    std::vector<unsigned char> buf(nxy * 8);
    for (int k = 0; k < 3; ++k) {
        const Var* v = nullptr;
        for (const Var& c : h.vars)
            if (c.name == names[k]) v = &c;
        if (!v || v->type != T_DOUBLE || v->dims.size() != 3) return MLQ_ERR_BADARG;
        // C order (z, y, x): the Fortran (x, y, z) array
        const bool rec = (int)v->dims[0] == h.recdim;
        const uint64_t len_z = rec ? h.numrecs : h.dim_len[v->dims[0]];
        if (len_z != (uint64_t)n3 || h.dim_len[v->dims[1]] != (uint64_t)n2 || h.dim_len[v->dims[2]] != (uint64_t)n1)
            return MLQ_ERR_BADARG;
        for (int z = 0; z < n3; ++z) {
            const uint64_t off = rec ? v->begin + (uint64_t)z * h.recsize : v->begin + (uint64_t)z * nxy * 8;
            if (std::fseek(g.f, (long)off, SEEK_SET) != 0) return MLQ_ERR_IO;
            if (std::fread(buf.data(), 1, buf.size(), g.f) != buf.size()) return MLQ_ERR_IO;
            get_be_doubles(buf.data(), nxy, u + ((size_t)k * n3 + z) * nxy);
        }
    }
    return MLQ_OK;
}

}  // extern "C"
