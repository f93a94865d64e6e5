// convert.cpp — the reference's graph-file converters (main.cu -m txt-bel,
// mtx-bel, tsv-bel, tsv-mtx, bel-mtx), host code.
//
// Each converter writes the same bytes as the reference's MtB_Writer method
// (include/FIleReader.cuh:456-912) for every input the reference handles.
// Where the reference has undefined behaviour or cannot finish (an empty
// input, an empty line in a .txt file, a missing size line), these return an
// error status instead; the differences are listed beside each function.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <utility>
#include <vector>

#include "internal.h"

namespace beep {
namespace {

using Pair32 = std::pair<uint32_t, uint32_t>;

struct File {
    FILE *fp = nullptr;
    ~File() {
        if (fp)
            std::fclose(fp);
    }
};

// .bel records {u64 dst, u64 src, u64 0} (FIleReader.cuh:437-445, 627-633).
template <typename P> beep_status write_bel_records(const char *path, const std::vector<P> &e, uint64_t *n_out) {
    File w;
    w.fp = std::fopen(path, "wb");
    if (!w.fp)
        return fail(BEEP_ERR_IO, std::string("cannot create ") + path);
    std::vector<uint64_t> buf;
    const size_t shard = 1 << 16;
    for (size_t i0 = 0; i0 < e.size(); i0 += shard) {
        const size_t i1 = std::min(e.size(), i0 + shard);
        buf.clear();
        for (size_t i = i0; i < i1; ++i) {
            buf.push_back((uint64_t)e[i].second);
            buf.push_back((uint64_t)e[i].first);
            buf.push_back(0);
        }
        if (std::fwrite(buf.data(), 8, buf.size(), w.fp) != buf.size())
            return fail(BEEP_ERR_IO, std::string("short write to ") + path);
    }
    if (n_out)
        *n_out = e.size();
    return BEEP_OK;
}

// "%%MatrixMarket matrix coordinate general", "n n m", then "src dst weight"
// per edge, n = source of the last edge (FIleReader.cuh:736-750, 789-810).
beep_status write_market(const char *path, const std::vector<Pair32> &e, const std::vector<int32_t> &wt,
                         uint64_t *n_out) {
    if (e.empty()) // the reference reads fileEdges[m - 1] here
        return fail(BEEP_ERR_PARSE, "no edges to convert");
    File w;
    w.fp = std::fopen(path, "w");
    if (!w.fp)
        return fail(BEEP_ERR_IO, std::string("cannot create ") + path);
    const unsigned long long n = e.back().first;
    std::fprintf(w.fp, "%%%%MatrixMarket matrix coordinate general\n%llu %llu %llu\n", n, n,
                 (unsigned long long)e.size());
    for (size_t i = 0; i < e.size(); ++i)
        std::fprintf(w.fp, "%u %u %d\n", e[i].first, e[i].second, wt[i]);
    if (std::ferror(w.fp))
        return fail(BEEP_ERR_IO, std::string("short write to ") + path);
    if (n_out)
        *n_out = e.size();
    return BEEP_OK;
}

// txt-bel: write_txt_bel<uint, uint>(src, dst, makeFull = true, numCol = 2,
// srcIndex = 0) (main.cu:64-66, FIleReader.cuh:816-907). '%' lines are
// skipped; a line whose first two fields parse as unsigned integers a != b
// adds (a, b) and (b, a), truncated to 32 bits; then sort and unique.
// Differences: an empty line is skipped (the reference's fscanf loop stops
// advancing there), lines of any length are read (the reference's buffer
// holds 99 characters).
beep_status txt_bel(const char *src, const char *dst, uint64_t *n_out) {
    std::ifstream in(src);
    if (!in)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + src);
    std::vector<Pair32> e;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '%')
            continue;
        unsigned long long a = 0, b = 0;
        if (std::sscanf(line.c_str(), "%llu %llu", &a, &b) == 2 && a != b) {
            e.emplace_back((uint32_t)a, (uint32_t)b);
            e.emplace_back((uint32_t)b, (uint32_t)a);
        }
    }
    std::sort(e.begin(), e.end());
    e.erase(std::unique(e.begin(), e.end()), e.end());
    return write_bel_records(dst, e, n_out);
}

// mtx-bel: write_market_bel<uint, int>(src, dst, makeFull = false)
// (main.cu:40-43, FIleReader.cuh:461-641). Comment lines set the banner flags,
// the last one winning; "rows cols nnz" (or "rows cols" for a dense array);
// then nnz entry lines, stopping at the first malformed one. Each entry adds
// (row, col) -- ids as written, not shifted -- and, in a symmetric file,
// (col, row) unless it is a loop. Sorted, duplicates and loops kept.
// Differences: a missing or malformed size line is an error (the reference
// goes on with uninitialised sizes); a non-square matrix is an error (the
// reference writes no file and exits 0).
beep_status mtx_bel(const char *src, const char *dst, uint64_t *n_out) {
    std::ifstream in(src);
    if (!in)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + src);
    bool symmetric = false, array = false, pattern = false;
    std::string line;
    bool have_size = false;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] != '%') {
            have_size = true;
            break;
        }
        if (line.size() >= 2) {
            symmetric = line.find("symmetric") != std::string::npos;
            array = line.find("array") != std::string::npos;
            pattern = line.find("pattern") != std::string::npos;
        }
    }
    long long nx = 0, ny = 0, nnz = 0;
    const int got = have_size ? std::sscanf(line.c_str(), "%lld %lld %lld", &nx, &ny, &nnz) : 0;
    if (array && got == 2)
        nnz = nx * ny;
    else if (!array && got == 3) {
        if (nx != ny)
            return fail(BEEP_ERR_PARSE, std::string(src) + ": not square");
    } else {
        return fail(BEEP_ERR_PARSE, std::string(src) + ": invalid problem description");
    }
    // the reference keeps both sizes in 32-bit unsigned variables
    const uint32_t nodes = (uint32_t)nx, entries = (uint32_t)nnz;
    std::vector<Pair32> e;
    for (unsigned long long i = 0; i < entries; ++i) {
        if (!std::getline(in, line))
            line.clear();
        long long r = 0, c = 0;
        double val = 0;
        int k;
        if (!pattern) {
            k = std::sscanf(line.c_str(), "%lld %lld %lf", &r, &c, &val);
            if (array && k == 1) {
                c = (long long)(i / nodes);
                r = (long long)(i - (unsigned long long)nodes * (unsigned long long)c);
            } else if (array || k < 2) {
                break;
            }
        } else {
            k = std::sscanf(line.c_str(), "%lld %lld", &r, &c);
            if (array && k == 1) {
                c = (long long)(i / nodes);
                r = (long long)(i - (unsigned long long)nodes * (unsigned long long)c);
            } else if (array || k != 2) {
                break;
            }
        }
        e.emplace_back((uint32_t)r, (uint32_t)c);
        if (symmetric && c != r)
            e.emplace_back((uint32_t)c, (uint32_t)r);
    }
    std::sort(e.begin(), e.end());
    return write_bel_records(dst, e, n_out);
}

// tsv-bel: write_tsv_bel<uint64, uint64> (main.cu:46-50,
// FIleReader.cuh:324-381): "dst src weight" triples until one fails to
// parse, written as records {dst, src, 0} in file order.
beep_status tsv_bel(const char *src, const char *dst, uint64_t *n_out) {
    File r;
    r.fp = std::fopen(src, "r");
    if (!r.fp)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + src);
    std::vector<std::pair<uint64_t, uint64_t>> e;
    unsigned long long d = 0, s = 0, w = 0;
    while (std::fscanf(r.fp, "%llu %llu %llu", &d, &s, &w) == 3)
        e.emplace_back((uint64_t)s, (uint64_t)d);
    return write_bel_records(dst, e, n_out);
}

// tsv-mtx: write_tsv_market<uint, int> (main.cu:52-56,
// FIleReader.cuh:706-753): "dst src weight" triples; ids truncated to 32 bits,
// the weight to its low 32 bits as a signed int (the reference scans it with
// %llu into an int).
beep_status tsv_mtx(const char *src, const char *dst, uint64_t *n_out) {
    File r;
    r.fp = std::fopen(src, "r");
    if (!r.fp)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + src);
    std::vector<Pair32> e;
    std::vector<int32_t> wt;
    unsigned long long d = 0, s = 0, w = 0;
    while (std::fscanf(r.fp, "%llu %llu %llu", &d, &s, &w) == 3) {
        e.emplace_back((uint32_t)s, (uint32_t)d);
        wt.push_back((int32_t)(uint32_t)w);
    }
    return write_market(dst, e, wt, n_out);
}

// bel-mtx: write_bel_market<uint, int> (main.cu:58-62,
// FIleReader.cuh:757-813): .bel records (a trailing partial record is
// ignored); ids truncated to 32 bits, the weight to the low 32 bits of its
// word as a signed int (the reference copies 8 bytes into an int).
beep_status bel_mtx(const char *src, const char *dst, uint64_t *n_out) {
    File r;
    r.fp = std::fopen(src, "rb");
    if (!r.fp)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + src);
    std::vector<Pair32> e;
    std::vector<int32_t> wt;
    uint64_t rec[3 * 1024];
    size_t got;
    while ((got = std::fread(rec, 24, 1024, r.fp)) > 0) {
        for (size_t i = 0; i < got; ++i) {
            e.emplace_back((uint32_t)rec[3 * i + 1], (uint32_t)rec[3 * i + 0]);
            wt.push_back((int32_t)(uint32_t)rec[3 * i + 2]);
        }
    }
    return write_market(dst, e, wt, n_out);
}

} // namespace
} // namespace beep

using namespace beep;

extern "C" beep_status beep_convert(beep_convert_task task, const char *src_path, const char *dst_path,
                                    uint64_t *records_out) {
    if (!src_path || !dst_path)
        return fail(BEEP_ERR_INVALID_ARG, "beep_convert: bad arguments");
    if (records_out)
        *records_out = 0;
    switch (task) {
    case BEEP_CONV_TXT_BEL:
        return txt_bel(src_path, dst_path, records_out);
    case BEEP_CONV_MTX_BEL:
        return mtx_bel(src_path, dst_path, records_out);
    case BEEP_CONV_TSV_BEL:
        return tsv_bel(src_path, dst_path, records_out);
    case BEEP_CONV_TSV_MTX:
        return tsv_mtx(src_path, dst_path, records_out);
    case BEEP_CONV_BEL_MTX:
        return bel_mtx(src_path, dst_path, records_out);
    }
    return fail(BEEP_ERR_INVALID_ARG, "beep_convert: unknown task");
}
