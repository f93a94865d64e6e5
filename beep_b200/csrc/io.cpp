// io.cpp — .bel / .mtx readers and writer, and deterministic synthetic graph
// generators (host code).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <numeric>
#include <sstream>

#include <omp.h>

#include "internal.h"

namespace beep {

// ---------------------------------------------------------------------------
// .bel: 24-byte records {u64 dst, u64 src, u64 weight}; src at byte 8, dst at
// byte 0 (include/FIleReader.cuh:63-89).
// ---------------------------------------------------------------------------
beep_status read_bel(const char *path, std::vector<uint32_t> &src, std::vector<uint32_t> &dst) {
    FILE *fp = std::fopen(path, "rb");
    if (!fp)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + path);
    std::fseek(fp, 0, SEEK_END);
    long long bytes = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (bytes < 0 || bytes % 24 != 0) {
        std::fclose(fp);
        return fail(BEEP_ERR_PARSE, std::string(path) + ": size is not a multiple of 24 bytes");
    }
    size_t ne = (size_t)(bytes / 24);
    std::vector<uint64_t> buf(3 * std::min<size_t>(ne, 1 << 20) + 3);
    src.resize(ne);
    dst.resize(ne);
    size_t done = 0;
    while (done < ne) {
        size_t chunk = std::min<size_t>(ne - done, 1 << 20);
        if (std::fread(buf.data(), 24, chunk, fp) != chunk) {
            std::fclose(fp);
            return fail(BEEP_ERR_IO, std::string(path) + ": short read");
        }
        for (size_t i = 0; i < chunk; ++i) {
            uint64_t d = buf[3 * i + 0], s = buf[3 * i + 1];
            if ((s >> 32) || (d >> 32)) {
                std::fclose(fp);
                return fail(BEEP_ERR_PARSE, std::string(path) + ": vertex id does not fit 32 bits");
            }
            src[done + i] = (uint32_t)s;
            dst[done + i] = (uint32_t)d;
        }
        done += chunk;
    }
    std::fclose(fp);
    return BEEP_OK;
}

// ---------------------------------------------------------------------------
// .mtx query files (include/FIleReader.cuh:130-212, 299-353): '%' comment
// lines, of which '%%' lines set symmetric/pattern/array; a "rows cols nnz"
// line; then 0-based "row col [value]" lines (not shifted to 0 from 1).
// Reading stops at the first line that does not parse, as read_market does.
// ---------------------------------------------------------------------------
beep_status read_mtx(const char *path, std::vector<int32_t> &src, std::vector<int32_t> &dst) {
    std::ifstream in(path);
    if (!in)
        return fail(BEEP_ERR_IO, std::string("cannot open ") + path);
    std::string line;
    bool symmetric = false, pattern = false, array = false;
    bool have_header = false;
    while (std::getline(in, line)) {
        if (!line.empty() && line[0] == '%') {
            if (line.size() >= 2 && line[1] == '%') {
                symmetric = line.find("symmetric") != std::string::npos;
                pattern = line.find("pattern") != std::string::npos;
                array = line.find("array") != std::string::npos;
            }
            continue;
        }
        have_header = true;
        break;
    }
    if (!have_header)
        return fail(BEEP_ERR_PARSE, std::string(path) + ": missing size line");
    long long rows = 0, cols = 0, nnz = 0;
    if (std::sscanf(line.c_str(), "%lld %lld %lld", &rows, &cols, &nnz) != 3)
        return fail(BEEP_ERR_PARSE, std::string(path) + ": invalid problem description");
    if (array)
        return fail(BEEP_ERR_PARSE, std::string(path) + ": dense array .mtx is not a graph");
    if (rows != cols)
        return fail(BEEP_ERR_PARSE, std::string(path) + ": matrix is not square");
    src.clear();
    dst.clear();
    while (std::getline(in, line)) {
        long long r = 0, c = 0;
        double val = 0;
        int got = pattern ? std::sscanf(line.c_str(), "%lld %lld", &r, &c)
                          : std::sscanf(line.c_str(), "%lld %lld %lf", &r, &c, &val);
        if (got < 2)
            break;
        if (r < 0 || c < 0 || r >= rows || c >= cols)
            return fail(BEEP_ERR_PARSE, std::string(path) + ": vertex id out of range in line '" + line + "'");
        src.push_back((int32_t)r);
        dst.push_back((int32_t)c);
        if (symmetric && r != c) {
            src.push_back((int32_t)c);
            dst.push_back((int32_t)r);
        }
    }
    if (src.empty())
        return fail(BEEP_ERR_PARSE, std::string(path) + ": no edges");
    return BEEP_OK;
}

// Query CSR as CSRCOO::from_edgelist builds it (include/CSRCOO.cuh:37-80):
// self loops dropped, n = largest source + 1, rows by source (the reference
// asserts sorted input; a stable sort accepts any order), file order kept
// within a row.
beep_status query_from_edges(const std::vector<int32_t> &src, const std::vector<int32_t> &dst, Query *q) {
    if (src.size() != dst.size())
        return fail(BEEP_ERR_INVALID_ARG, "query src/dst sizes differ");
    std::vector<std::pair<int32_t, int32_t>> e;
    int32_t n = 0;
    for (size_t i = 0; i < src.size(); ++i) {
        if (src[i] < 0 || dst[i] < 0)
            return fail(BEEP_ERR_INVALID_ARG, "negative query vertex id");
        if (src[i] == dst[i])
            continue;
        e.emplace_back(src[i], dst[i]);
        n = std::max(n, src[i] + 1);
    }
    if (e.empty())
        return fail(BEEP_ERR_UNSUPPORTED, "query has no edges");
    for (auto &x : e)
        if (x.second >= n)
            return fail(BEEP_ERR_UNSUPPORTED, "query edge points past the last source vertex");
    if (n > kMaxQ)
        return fail(BEEP_ERR_UNSUPPORTED, "query has more than " + std::to_string(kMaxQ) + " vertices");
    std::stable_sort(e.begin(), e.end(), [](auto &a, auto &b) { return a.first < b.first; });
    q->qn = n;
    q->row_ptr.assign(n + 1, 0);
    q->col.clear();
    for (auto &x : e) {
        q->row_ptr[x.first + 1]++;
        q->col.push_back(x.second);
    }
    for (int32_t v = 0; v < n; ++v)
        q->row_ptr[v + 1] += q->row_ptr[v];
    return BEEP_OK;
}

} // namespace beep

// ---------------------------------------------------------------------------
// synthetic generators
// ---------------------------------------------------------------------------
namespace {

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Counter-based stream: value i of stream (seed, key).
struct Stream {
    uint64_t base, i = 0;
    Stream(uint64_t seed, uint64_t key) : base(splitmix64(seed ^ splitmix64(key + 0x632BE59BD9B4E019ull))) {}
    uint64_t next() { return splitmix64(base + 0x9E3779B97F4A7C15ull * (++i)); }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); } // [0,1)
};

// Undirected simple graph from an edge list: drop loops, add both
// directions, sort rows, remove duplicates.
beep_status to_csr(int64_t n, std::vector<std::pair<uint32_t, uint32_t>> &und, int64_t *n_out, int64_t *m_out,
                   int32_t *row_ptr, int32_t *col_ind) {
    std::vector<int64_t> cnt(n + 1, 0);
    for (auto &e : und)
        if (e.first != e.second) {
            cnt[e.first + 1]++;
            cnt[e.second + 1]++;
        }
    for (int64_t v = 0; v < n; ++v)
        cnt[v + 1] += cnt[v];
    std::vector<uint32_t> adj(cnt[n]);
    std::vector<int64_t> fillp(cnt.begin(), cnt.end() - 1);
    for (auto &e : und)
        if (e.first != e.second) {
            adj[fillp[e.first]++] = e.second;
            adj[fillp[e.second]++] = e.first;
        }
    std::vector<int64_t> deg(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < n; ++v) {
        auto b = adj.begin() + cnt[v], e = adj.begin() + cnt[v + 1];
        std::sort(b, e);
        deg[v] = std::unique(b, e) - b;
    }
    int64_t m = 0;
    for (int64_t v = 0; v < n; ++v)
        m += deg[v];
    if (m >= (int64_t)1 << 31)
        return beep::fail(BEEP_ERR_UNSUPPORTED, "generated graph exceeds int32 CSR");
    *n_out = n;
    *m_out = m;
    if (row_ptr && col_ind) {
        int64_t off = 0;
        for (int64_t v = 0; v < n; ++v) {
            row_ptr[v] = (int32_t)off;
            std::copy(adj.begin() + cnt[v], adj.begin() + cnt[v] + deg[v], col_ind + off);
            off += deg[v];
        }
        row_ptr[n] = (int32_t)off;
    }
    return BEEP_OK;
}

} // namespace

extern "C" beep_status beep_gen_erdos_renyi(int64_t n, double p, uint64_t seed, int64_t *n_out, int64_t *m_out,
                                            int32_t *row_ptr, int32_t *col_ind) {
    if (n <= 0 || n > (1ll << 31) || !(p >= 0.0 && p <= 1.0) || !n_out || !m_out)
        return beep::fail(BEEP_ERR_INVALID_ARG, "beep_gen_erdos_renyi: bad arguments");
    // Row u draws its neighbours v > u by geometric skips from stream (seed, u).
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> parts(omp_get_max_threads());
#pragma omp parallel
    {
        auto &out = parts[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 256)
        for (int64_t u = 0; u < n; ++u) {
            if (p <= 0.0)
                continue;
            Stream s(seed, (uint64_t)u);
            int64_t v = u;
            const double lq = std::log1p(-p);
            for (;;) {
                int64_t skip = 0;
                if (p < 1.0) {
                    double r = s.uniform();
                    skip = (int64_t)std::floor(std::log1p(-r) / lq);
                }
                v += skip + 1;
                if (v >= n)
                    break;
                out.emplace_back((uint32_t)u, (uint32_t)v);
            }
        }
    }
    std::vector<std::pair<uint32_t, uint32_t>> und;
    for (auto &pt : parts)
        und.insert(und.end(), pt.begin(), pt.end());
    return to_csr(n, und, n_out, m_out, row_ptr, col_ind);
}

extern "C" beep_status beep_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                                     int64_t *n_out, int64_t *m_out, int32_t *row_ptr, int32_t *col_ind) {
    if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 || !n_out ||
        !m_out)
        return beep::fail(BEEP_ERR_INVALID_ARG, "beep_gen_rmat: bad arguments");
    const int64_t n = 1ll << scale;
    const int64_t ne = (int64_t)edge_factor << scale;
    std::vector<std::pair<uint32_t, uint32_t>> und(ne);
    const double ab = a + b, abc = a + b + c;
    // Edge e descends `scale` levels of the (a,b,c,d) quadrant recursion using
    // stream (seed, e).
#pragma omp parallel for schedule(static, 4096)
    for (int64_t e = 0; e < ne; ++e) {
        Stream s(seed, (uint64_t)e);
        uint32_t u = 0, v = 0;
        for (int l = 0; l < scale; ++l) {
            double r = s.uniform();
            uint32_t bu = 0, bv = 0;
            if (r < a) {
            } else if (r < ab) {
                bv = 1;
            } else if (r < abc) {
                bu = 1;
            } else {
                bu = 1;
                bv = 1;
            }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        und[e] = {u, v};
    }
    return to_csr(n, und, n_out, m_out, row_ptr, col_ind);
}

extern "C" beep_status beep_gen_chung_lu(int64_t n, double avg_degree, double exponent, uint64_t seed,
                                         int64_t *n_out, int64_t *m_out, int32_t *row_ptr, int32_t *col_ind) {
    if (n <= 1 || n > (1ll << 31) || !(avg_degree > 0) || !(exponent > 1.0) || !n_out || !m_out)
        return beep::fail(BEEP_ERR_INVALID_ARG, "beep_gen_chung_lu: bad arguments");
    // Expected degree of vertex i proportional to (i+1)^(-1/(exponent-1));
    // m = n*avg/2 edges, each endpoint drawn by weight (inverse CDF).
    std::vector<double> cdf(n);
    double acc = 0;
    const double ex = -1.0 / (exponent - 1.0);
    for (int64_t i = 0; i < n; ++i) {
        acc += std::pow((double)(i + 1), ex);
        cdf[i] = acc;
    }
    for (auto &x : cdf)
        x /= acc;
    const int64_t ne = (int64_t)std::llround((double)n * avg_degree / 2.0);
    std::vector<std::pair<uint32_t, uint32_t>> und(ne);
#pragma omp parallel for schedule(static, 4096)
    for (int64_t e = 0; e < ne; ++e) {
        Stream s(seed, (uint64_t)e);
        double r1 = s.uniform(), r2 = s.uniform();
        uint32_t u = (uint32_t)(std::lower_bound(cdf.begin(), cdf.end(), r1) - cdf.begin());
        uint32_t v = (uint32_t)(std::lower_bound(cdf.begin(), cdf.end(), r2) - cdf.begin());
        if (u >= n)
            u = (uint32_t)(n - 1);
        if (v >= n)
            v = (uint32_t)(n - 1);
        und[e] = {u, v};
    }
    return to_csr(n, und, n_out, m_out, row_ptr, col_ind);
}

extern "C" beep_status beep_write_bel(const char *path, int64_t n, const int32_t *row_ptr, const int32_t *col_ind) {
    if (!path || n < 0 || !row_ptr || (!col_ind && row_ptr[n] > 0))
        return beep::fail(BEEP_ERR_INVALID_ARG, "beep_write_bel: bad arguments");
    FILE *fp = std::fopen(path, "wb");
    if (!fp)
        return beep::fail(BEEP_ERR_IO, std::string("cannot create ") + path);
    std::vector<uint64_t> buf;
    buf.reserve(3 * 65536);
    for (int64_t v = 0; v < n; ++v) {
        for (int64_t e = row_ptr[v]; e < row_ptr[v + 1]; ++e) {
            buf.push_back((uint64_t)(uint32_t)col_ind[e]); // dst at byte 0
            buf.push_back((uint64_t)v);                    // src at byte 8
            buf.push_back(0);                              // weight
            if (buf.size() >= 3 * 65536) {
                if (std::fwrite(buf.data(), 8, buf.size(), fp) != buf.size()) {
                    std::fclose(fp);
                    return beep::fail(BEEP_ERR_IO, std::string("short write to ") + path);
                }
                buf.clear();
            }
        }
    }
    if (!buf.empty() && std::fwrite(buf.data(), 8, buf.size(), fp) != buf.size()) {
        std::fclose(fp);
        return beep::fail(BEEP_ERR_IO, std::string("short write to ") + path);
    }
    std::fclose(fp);
    return BEEP_OK;
}
