#include "csc.hpp"

#include <omp.h>

#include <parallel/algorithm>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "blest.h"

namespace blest {

double Csc::average_degree() const {
    double average = 0;
    for (uint32_t j = 0; j < n; ++j) average += degree(j);
    return n ? average / n : 0.0;
}

uint32_t Csc::max_degree() const {
    uint32_t m = 0;
    for (uint32_t j = 0; j < n; ++j) m = std::max(m, degree(j));
    return m;
}

uint32_t Csc::max_bandwidth() const {
    uint32_t band = 0;
    for (uint32_t j = 0; j < n; ++j) {
        if (col_ptrs[j] == col_ptrs[j + 1]) continue;
        int64_t d = (int64_t)j - (int64_t)rows[col_ptrs[j + 1] - 1];
        band = std::max<uint32_t>(band, (uint32_t)(d < 0 ? -d : d));
    }
    return band;
}

double Csc::average_bandwidth() const {
    double average = 0;
    for (uint32_t j = 0; j < n; ++j) {
        if (col_ptrs[j] == col_ptrs[j + 1]) continue;
        int64_t d = (int64_t)j - (int64_t)rows[col_ptrs[j + 1] - 1];
        average += (uint32_t)(d < 0 ? -d : d);
    }
    return n ? average / n : 0.0;
}

// Restatement of Common.cuh:100-250. The floating-point operations are
// kept in the reference's order so the decision is the same on the same
// degree sequence.
bool is_social_degree_distribution(const std::vector<uint32_t>& deg) {
    const uint32_t n = (uint32_t)deg.size();
    if (n == 0) return false;
    uint32_t maxDeg = 0;
    unsigned long long sumDeg = 0;
    for (uint32_t d : deg) {
        sumDeg += d;
        maxDeg = std::max(maxDeg, d);
    }
    if (maxDeg == 0 || sumDeg == 0) return false;

    std::vector<uint32_t> sorted = deg;
    __gnu_parallel::sort(sorted.begin(), sorted.end());
    auto shareTop = [&](double frac) {
        double raw = frac * (double)n;
        uint32_t k = (uint32_t)std::ceil(raw);
        if (k == 0) k = 1;
        if (k > n) k = n;
        unsigned long long top = 0;
        for (uint32_t i = 0; i < k; ++i) top += sorted[n - 1 - i];
        return (double)top / (double)sumDeg;
    };
    const bool heavyTail = shareTop(0.01) >= 0.05 && shareTop(0.10) >= 0.40;

    std::vector<uint32_t> freq((size_t)maxDeg + 1, 0);
    for (uint32_t d : deg) ++freq[d];
    std::vector<double> xs, ys;
    for (uint32_t k = 5; k <= maxDeg; ++k) {
        if (freq[k] != 0) {
            xs.push_back(std::log((double)k));
            ys.push_back(std::log((double)freq[k]));
        }
    }
    bool powerLaw = false;
    const uint32_t m = (uint32_t)xs.size();
    if (m >= 3u) {
        double sx = 0, sy = 0, sxy = 0, sxx = 0;
        for (uint32_t i = 0; i < m; ++i) {
            sx += xs[i];
            sy += ys[i];
            sxy += xs[i] * ys[i];
            sxx += xs[i] * xs[i];
        }
        const double nd = (double)m;
        const double denom = nd * sxx - sx * sx;
        if (denom > 0.0) {
            const double slope = (nd * sxy - sx * sy) / denom;
            const double intercept = (sy - slope * sx) / nd;
            const double yMean = sy / nd;
            double ssTot = 0, ssRes = 0;
            for (uint32_t i = 0; i < m; ++i) {
                const double yHat = intercept + slope * xs[i];
                ssTot += (ys[i] - yMean) * (ys[i] - yMean);
                ssRes += (ys[i] - yHat) * (ys[i] - yHat);
            }
            if (ssTot > 0.0) {
                const double r2 = 1.0 - ssRes / ssTot;
                const double gamma = -slope;
                powerLaw = r2 >= 0.70 && gamma >= 1.0 && gamma <= 5.0;
            }
        }
    }
    return heavyTail || powerLaw;
}

bool classify_social(const Csc& g) {
    std::vector<uint32_t> outDeg(g.n), inDeg(g.n, 0);
    for (uint32_t j = 0; j < g.n; ++j) outDeg[j] = g.degree(j);
    // in-degrees without atomics: each thread counts the rows of its range
#pragma omp parallel
    {
        const uint32_t T = (uint32_t)omp_get_num_threads(), me = (uint32_t)omp_get_thread_num();
        const uint32_t lo = (uint32_t)((uint64_t)g.n * me / T), hi = (uint32_t)((uint64_t)g.n * (me + 1) / T);
        for (uint32_t p = 0; p < g.nnz; ++p)
            if (g.rows[p] - lo < hi - lo) ++inDeg[g.rows[p]];
    }
    bool social = is_social_degree_distribution(inDeg) || is_social_degree_distribution(outDeg);
    return social || (g.average_degree() > kSocialThreshold);
}

static void sort_columns(Csc& g) {
#pragma omp parallel for schedule(dynamic, 2048)
    for (int64_t j = 0; j < (int64_t)g.n; ++j)
        std::sort(g.rows.begin() + g.col_ptrs[j], g.rows.begin() + g.col_ptrs[j + 1]);
}

namespace {

inline bool mtx_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Unsigned decimal token at buf[p] (after whitespace); false if it is not one.
inline bool mtx_uint(const char* buf, size_t size, size_t& p, uint64_t& out) {
    while (p < size && mtx_space(buf[p])) ++p;
    if (p < size && buf[p] == '+') ++p;
    if (p >= size || buf[p] < '0' || buf[p] > '9') return false;
    uint64_t v = 0;
    while (p < size && buf[p] >= '0' && buf[p] <= '9') {
        v = v * 10 + (uint64_t)(buf[p] - '0');
        ++p;
    }
    out = v;
    return p >= size || mtx_space(buf[p]);
}

// A numeric value token at buf[p] (after whitespace); false if there is none.
inline bool mtx_value(const char* buf, size_t size, size_t& p) {
    while (p < size && mtx_space(buf[p])) ++p;
    if (p >= size) return false;
    char* e = nullptr;
    std::strtod(buf + p, &e);
    if (e == buf + p || (e < buf + size && !mtx_space(*e))) return false;
    p = (size_t)(e - buf);
    return true;
}

// CSC with sorted columns (duplicates kept) from per-thread lists of packed
// (column << 32 | row) pairs: pairs are bucketed by column partition, then
// every partition counts, fills and sorts its own columns.
Csc csc_from_column_pairs(uint32_t n, std::vector<std::vector<uint64_t>>& parts) {
    uint32_t shift = 0;
    while (((uint64_t)n >> shift) > 4096) ++shift;
    const uint32_t P = n ? (uint32_t)((((uint64_t)n - 1) >> shift) + 1) : 1;
    const int T = (int)parts.size();
    std::vector<uint64_t> off((size_t)T * P, 0), pbase((size_t)P + 1, 0);
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < T; ++t)
        for (uint64_t x : parts[t]) ++off[(size_t)t * P + (uint32_t)(x >> (32 + shift))];
    uint64_t total = 0;
    for (uint32_t q = 0; q < P; ++q) {
        pbase[q] = total;
        for (int t = 0; t < T; ++t) {
            const uint64_t c = off[(size_t)t * P + q];
            off[(size_t)t * P + q] = total;
            total += c;
        }
    }
    pbase[P] = total;
    if (total > 0xFFFFFFFFull) throw Error(BLEST_ERR_UNSUPPORTED, "more than 2^32-1 non-zeros");
    std::vector<uint64_t> pairs(total);
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        uint64_t* o = off.data() + (size_t)t * P;
        for (uint64_t x : parts[t]) pairs[o[(uint32_t)(x >> (32 + shift))]++] = x;
        std::vector<uint64_t>().swap(parts[t]);
    }
    Csc g;
    g.n = n;
    g.nnz = (uint32_t)total;
    g.col_ptrs.assign((size_t)n + 1, 0);
    g.rows.resize(total);
    // column counts, each partition over its own pairs
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t qq = 0; qq < (int64_t)P; ++qq)
        for (uint64_t i = pbase[qq]; i < pbase[qq + 1]; ++i) ++g.col_ptrs[(uint32_t)(pairs[i] >> 32) + 1];
    for (uint32_t j = 0; j < n; ++j) g.col_ptrs[j + 1] += g.col_ptrs[j];
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t qq = 0; qq < (int64_t)P; ++qq) {
        const uint32_t q = (uint32_t)qq;
        const uint32_t lo = q << shift, hi = (uint32_t)std::min<uint64_t>(n, ((uint64_t)q + 1) << shift);
        if (lo >= hi) continue;
        std::vector<uint32_t> cur(g.col_ptrs.begin() + lo, g.col_ptrs.begin() + hi);
        for (uint64_t i = pbase[q]; i < pbase[q + 1]; ++i) {
            const uint64_t x = pairs[i];
            g.rows[cur[(uint32_t)(x >> 32) - lo]++] = (uint32_t)x;
        }
        for (uint32_t j = lo; j < hi; ++j) std::sort(g.rows.begin() + g.col_ptrs[j], g.rows.begin() + g.col_ptrs[j + 1]);
    }
    return g;
}

}  // namespace

// The reference's reader (CSC.cuh:98-185) as a parallel parser with the same
// token semantics as its stream loop: leading '%' lines skipped, then
// whitespace-separated tokens "n n' entries" and per entry "j i" (+ a value
// unless the matrix is a pattern); an entry j i adds row i-1 to column j-1
// (and column i-1 gets row j-1 when undirected); self loops are dropped
// before the range check; duplicates are kept; columns end sorted. The file
// is read whole and cut into per-thread chunks at token boundaries; a
// thread takes the entries whose first token lies in its chunk (reading on
// past its end to finish the last one), so token k of the body is entry
// k / tokens-per-entry whatever the chunking.
Csc csc_read_mtx(const std::string& path, bool undirected, bool binary) {
    std::ifstream file(path, std::ios::binary);
    if (!file.is_open()) throw Error(BLEST_ERR_IO, "cannot open Matrix Market file: " + path);
    file.seekg(0, std::ios::end);
    const size_t size = (size_t)file.tellg();
    file.seekg(0);
    std::vector<char> data(size + 1, '\0');
    if (size && !file.read(data.data(), (std::streamsize)size)) throw Error(BLEST_ERR_IO, "short read from " + path);
    const char* buf = data.data();
    size_t pos = 0;
    while (pos < size && buf[pos] == '%') {
        while (pos < size && buf[pos] != '\n') ++pos;
        if (pos < size) ++pos;
    }
    uint64_t n64 = 0, n2 = 0, lines = 0;
    if (!mtx_uint(buf, size, pos, n64) || !mtx_uint(buf, size, pos, n2) || !mtx_uint(buf, size, pos, lines) ||
        n64 > 0xFFFFFFFFull)
        throw Error(BLEST_ERR_IO, "bad Matrix Market size line: " + path);
    const uint32_t n = (uint32_t)n64;
    const uint32_t K = binary ? 2 : 3;  // tokens per entry
    const int T = std::max(1, omp_get_max_threads());
    // chunk t = [cut[t], cut[t+1]), each cut moved forward to a token boundary
    std::vector<size_t> cut((size_t)T + 1);
    for (int t = 0; t <= T; ++t) {
        size_t c = pos + (size - pos) * (size_t)t / (size_t)T;
        while (t > 0 && c < size && c > pos && !mtx_space(buf[c - 1])) ++c;
        cut[t] = std::min(c, size);
    }
    cut[T] = size;
    std::vector<uint64_t> tok((size_t)T + 1, 0);  // token starts per chunk, then prefix
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; ++t) {
        uint64_t c = 0;
        for (size_t p = cut[t]; p < cut[t + 1]; ++p)
            c += !mtx_space(buf[p]) && (p == pos || mtx_space(buf[p - 1]));
        tok[t + 1] = c;
    }
    for (int t = 0; t < T; ++t) tok[t + 1] += tok[t];
    // first failing entry (sequential reading order) and its message
    std::vector<uint64_t> badAt((size_t)T, ~0ull);
    std::vector<int> badKind((size_t)T, 0);  // 1 truncated, 2 missing value, 3 index out of range
    std::vector<std::vector<uint64_t>> parts((size_t)T);
#pragma omp parallel for schedule(static, 1) num_threads(T)
    for (int t = 0; t < T; ++t) {
        std::vector<uint64_t>& out = parts[t];
        uint64_t k = tok[t];
        size_t p = cut[t];
        while (k < (uint64_t)lines * K) {
            // next token start in this chunk
            while (p < cut[t + 1] && mtx_space(buf[p])) ++p;
            if (p >= cut[t + 1]) break;
            if (k % K != 0) {  // a token of an entry begun in the previous chunk
                while (p < size && !mtx_space(buf[p])) ++p;
                ++k;
                continue;
            }
            const uint64_t entry = k / K;
            uint64_t j = 0, i = 0;
            size_t q = p;
            int bad = 0;
            if (!mtx_uint(buf, size, q, j) || !mtx_uint(buf, size, q, i)) bad = 1;
            else if (!binary && !mtx_value(buf, size, q)) bad = 2;
            else if (i != j && (i == 0 || j == 0 || i > n || j > n)) bad = 3;
            if (bad) {
                badAt[t] = entry;
                badKind[t] = bad;
                break;
            }
            if (i != j) {
                out.push_back(((j - 1) << 32) | (i - 1));
                if (undirected) out.push_back(((i - 1) << 32) | (j - 1));
            }
            // step past this entry's first token only; its other tokens are
            // skipped above as non-first tokens (they may lie in the next chunk)
            while (p < size && !mtx_space(buf[p])) ++p;
            ++k;
        }
    }
    int t0 = -1;
    for (int t = 0; t < T; ++t)
        if (badAt[t] != ~0ull && (t0 < 0 || badAt[t] < badAt[t0])) t0 = t;
    if (t0 < 0 && tok[T] < (uint64_t)lines * K) throw Error(BLEST_ERR_IO, "truncated Matrix Market file: " + path);
    if (t0 >= 0) {
        if (badKind[t0] == 2) throw Error(BLEST_ERR_IO, "missing value in Matrix Market entry: " + path);
        if (badKind[t0] == 3) throw Error(BLEST_ERR_IO, "Matrix Market index out of range: " + path);
        throw Error(BLEST_ERR_IO, "truncated Matrix Market file: " + path);
    }
    Csc g = csc_from_column_pairs(n, parts);
    g.is_social = classify_social(g);
    return g;
}

Csc csc_read_mtx_auto(const std::string& path) {
    std::ifstream file(path);
    if (!file.is_open()) throw Error(BLEST_ERR_IO, "cannot open Matrix Market file: " + path);
    std::string banner;
    std::getline(file, banner);
    std::string lower = banner;
    std::transform(lower.begin(), lower.end(), lower.begin(), ::tolower);
    const bool binary = lower.find("pattern") != std::string::npos;
    const bool undirected = lower.find("symmetric") != std::string::npos ||
                            lower.find("hermitian") != std::string::npos;
    file.close();
    return csc_read_mtx(path, undirected, binary);
}

void csc_save_bin(const Csc& g, const std::string& path) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw Error(BLEST_ERR_IO, "cannot write " + path);
    const uint8_t social = g.is_social ? 1 : 0;
    out.write((const char*)&g.n, 4);
    out.write((const char*)&g.nnz, 4);
    out.write((const char*)&social, 1);
    out.write((const char*)g.col_ptrs.data(), 4ull * (g.n + 1ull));
    out.write((const char*)g.rows.data(), 4ull * g.nnz);
    if (!out) throw Error(BLEST_ERR_IO, "short write to " + path);
}

Csc csc_load_bin(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw Error(BLEST_ERR_IO, "cannot open " + path);
    in.seekg(0, std::ios::end);
    const uint64_t size = (uint64_t)in.tellg();
    in.seekg(0);
    Csc g;
    uint8_t social = 0;
    in.read((char*)&g.n, 4);
    in.read((char*)&g.nnz, 4);
    in.read((char*)&social, 1);
    if (!in || size != 9ull + 4ull * (g.n + 1ull) + 4ull * g.nnz)
        throw Error(BLEST_ERR_IO, "corrupt or truncated CSC cache: " + path);
    g.is_social = social != 0;
    g.col_ptrs.resize((size_t)g.n + 1);
    g.rows.resize(g.nnz);
    in.read((char*)g.col_ptrs.data(), 4ull * (g.n + 1ull));
    in.read((char*)g.rows.data(), 4ull * g.nnz);
    if (!in) throw Error(BLEST_ERR_IO, "short read from " + path);
    if (g.col_ptrs[0] != 0 || g.col_ptrs[g.n] != g.nnz) throw Error(BLEST_ERR_IO, "inconsistent CSC cache: " + path);
    for (uint32_t j = 0; j < g.n; ++j)
        if (g.col_ptrs[j] > g.col_ptrs[j + 1]) throw Error(BLEST_ERR_IO, "inconsistent CSC cache: " + path);
    for (uint32_t p = 0; p < g.nnz; ++p)
        if (g.rows[p] >= g.n) throw Error(BLEST_ERR_IO, "row index out of range in CSC cache: " + path);
    return g;
}

void ordering_save_bin(const std::vector<uint32_t>& inv, const std::string& path) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw Error(BLEST_ERR_IO, "cannot write " + path);
    out.write((const char*)inv.data(), 4ull * inv.size());
    if (!out) throw Error(BLEST_ERR_IO, "short write to " + path);
}

std::vector<uint32_t> ordering_load_bin(const std::string& path, uint32_t n) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw Error(BLEST_ERR_IO, "cannot open " + path);
    in.seekg(0, std::ios::end);
    if ((uint64_t)in.tellg() != 4ull * n) throw Error(BLEST_ERR_IO, "ordering cache size mismatch: " + path);
    in.seekg(0);
    std::vector<uint32_t> inv(n);
    in.read((char*)inv.data(), 4ull * n);
    if (!in) throw Error(BLEST_ERR_IO, "short read from " + path);
    if (!permutation_check(inv, n)) throw Error(BLEST_ERR_IO, "ordering cache is not a permutation: " + path);
    return inv;
}

// Parallel without atomics or sorting: thread t owns the rows of range t
// and scans every column in increasing order, counting (then writing) only
// the entries of its rows, so each transposed list is filled in increasing
// column order, as the sequential loop does.
Csc csc_transpose(const Csc& g) {
    Csc t;
    t.n = g.n;
    t.nnz = g.nnz;
    t.is_social = g.is_social;
    t.col_ptrs.assign((size_t)g.n + 1, 0);
    t.rows.resize(g.nnz);
    const uint32_t n = g.n;
    const uint32_t* rows = g.rows.data();
    const uint32_t* cp = g.col_ptrs.data();
    uint32_t* tp = t.col_ptrs.data();
    uint32_t* tr = t.rows.data();
#pragma omp parallel
    {
        const uint32_t T = (uint32_t)omp_get_num_threads(), me = (uint32_t)omp_get_thread_num();
        const uint32_t lo = (uint32_t)((uint64_t)n * me / T), hi = (uint32_t)((uint64_t)n * (me + 1) / T);
        const uint32_t span = hi - lo;
        for (uint32_t p = 0; p < g.nnz; ++p)
            if (rows[p] - lo < span) ++tp[rows[p] + 1];
#pragma omp barrier
#pragma omp single
        for (uint32_t i = 1; i <= n; ++i) tp[i] += tp[i - 1];
        std::vector<uint32_t> cursor(tp + lo, tp + hi);
        for (uint32_t j = 0; j < n; ++j)
            for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
                const uint32_t r = rows[p] - lo;
                if (r < span) tr[cursor[r]++] = j;
            }
    }
    return t;
}

// Every off-diagonal (i, j) has its (j, i): columns checked in parallel
// (binary search in the sorted column i), stopping early on the first miss.
bool csc_check_symmetry(const Csc& g) {
    int ok = 1;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t jj = 0; jj < (int64_t)g.n; ++jj) {
        if (!__atomic_load_n(&ok, __ATOMIC_RELAXED)) continue;
        const uint32_t j = (uint32_t)jj;
        for (uint32_t p = g.col_ptrs[j]; p < g.col_ptrs[j + 1]; ++p) {
            const uint32_t i = g.rows[p];
            if (i == j) continue;
            const auto b = g.rows.begin() + g.col_ptrs[i], e = g.rows.begin() + g.col_ptrs[i + 1];
            if (!std::binary_search(b, e, j)) {
                __atomic_store_n(&ok, 0, __ATOMIC_RELAXED);
                break;
            }
        }
    }
    return ok != 0;
}

Csc csc_symmetrize(const Csc& g) {
    std::vector<std::vector<uint32_t>> cols(g.n);
    for (uint32_t j = 0; j < g.n; ++j) {
        for (uint32_t p = g.col_ptrs[j]; p < g.col_ptrs[j + 1]; ++p) {
            const uint32_t i = g.rows[p];
            cols[j].push_back(i);
            if (i != j) cols[i].push_back(j);
        }
    }
    Csc s;
    s.n = g.n;
    s.is_social = g.is_social;
    s.col_ptrs.assign((size_t)g.n + 1, 0);
    uint64_t nnz = 0;
    for (uint32_t j = 0; j < g.n; ++j) {
        auto& v = cols[j];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        nnz += v.size();
        s.col_ptrs[j + 1] = (uint32_t)nnz;
    }
    s.nnz = (uint32_t)nnz;
    s.rows.resize(nnz);
    for (uint32_t j = 0; j < g.n; ++j) std::copy(cols[j].begin(), cols[j].end(), s.rows.begin() + s.col_ptrs[j]);
    return s;
}

bool permutation_check(const std::vector<uint32_t>& inv, uint32_t n) {
    if (inv.size() != n) return false;
    std::vector<uint8_t> seen(n, 0);
    for (uint32_t v : inv) {
        if (v >= n || seen[v]) return false;
        seen[v] = 1;
    }
    return true;
}

void csc_apply_permutation(Csc& g, const std::vector<uint32_t>& inv) {
    if (!permutation_check(inv, g.n)) throw Error(BLEST_ERR_INVALID_ARG, "Permutation check has failed.");
    std::vector<uint32_t> ptrs((size_t)g.n + 1, 0);
    for (uint32_t old = 0; old < g.n; ++old) ptrs[inv[old] + 1] = g.degree(old);
    for (uint32_t j = 0; j < g.n; ++j) ptrs[j + 1] += ptrs[j];
    std::vector<uint32_t> rows(g.nnz);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t old = 0; old < (int64_t)g.n; ++old) {
        const uint32_t nc = inv[old];
        uint32_t* dst = rows.data() + ptrs[nc];
        const uint32_t b = g.col_ptrs[old], e = g.col_ptrs[old + 1];
        for (uint32_t p = b; p < e; ++p) dst[p - b] = inv[g.rows[p]];
        std::sort(dst, dst + (e - b));
    }
    g.col_ptrs.swap(ptrs);
    g.rows.swap(rows);
}

// Symmetrised, de-duplicated, self-loop-free CSC of an edge stream, built
// without random-access atomics: the edges are drawn twice per thread (each
// thread a fixed range of edge indices) — once to count both directions per
// vertex partition (a few thousand consecutive-id partitions), once to write
// them as packed (vertex, neighbour) pairs into their partition's slice of
// one buffer — and each partition then fills, sorts and de-duplicates its
// own columns with counters that stay in cache. Columns are sorted and
// unique, so the arrays do not depend on the thread count or write order.
Csc csc_from_undirected_edges(uint32_t n, uint64_t m, const EdgeFn& edge) {
    uint32_t shift = 0;  // partition of vertex u: u >> shift, at most 4096 partitions
    while (((uint64_t)n >> shift) > 4096) ++shift;
    const uint32_t P = (uint32_t)((((uint64_t)n - 1) >> shift) + 1);
    const int T = omp_get_max_threads();
    std::vector<uint64_t> cnt((size_t)T * P, 0);  // [thread][partition]
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const uint64_t e0 = m * t / nt, e1 = m * (t + 1) / nt;
        uint64_t* c = cnt.data() + (size_t)t * P;
        for (uint64_t e = e0; e < e1; ++e) {
            uint32_t u, v;
            if (!edge(e, &u, &v) || u == v) continue;
            ++c[u >> shift];
            ++c[v >> shift];
        }
    }
    // partition-major offsets: partition p's pairs, thread by thread
    std::vector<uint64_t> off((size_t)T * P, 0), pbase((size_t)P + 1, 0);
    uint64_t total = 0;
    for (uint32_t p = 0; p < P; ++p) {
        pbase[p] = total;
        for (int t = 0; t < T; ++t) {
            off[(size_t)t * P + p] = total;
            total += cnt[(size_t)t * P + p];
        }
    }
    pbase[P] = total;
    std::vector<uint64_t> pairs(total);
#pragma omp parallel num_threads(T)
    {
        const int t = omp_get_thread_num(), nt = omp_get_num_threads();
        const uint64_t e0 = m * t / nt, e1 = m * (t + 1) / nt;
        uint64_t* o = off.data() + (size_t)t * P;
        for (uint64_t e = e0; e < e1; ++e) {
            uint32_t u, v;
            if (!edge(e, &u, &v) || u == v) continue;
            pairs[o[u >> shift]++] = ((uint64_t)u << 32) | v;
            pairs[o[v >> shift]++] = ((uint64_t)v << 32) | u;
        }
    }
    // per partition: neighbours of each of its columns, sorted and unique,
    // left in place at the front of the column's range of `pairs`
    std::vector<uint32_t> deg((size_t)n, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t pp = 0; pp < (int64_t)P; ++pp) {
        const uint32_t p = (uint32_t)pp;
        const uint32_t lo = p << shift, hi = (uint32_t)std::min<uint64_t>(n, ((uint64_t)p + 1) << shift);
        const uint32_t w = hi - lo;
        const uint64_t b = pbase[p], e = pbase[p + 1];
        std::vector<uint64_t> start((size_t)w + 1, 0);  // column j - lo occupies [start[j-lo], start[j-lo+1])
        for (uint64_t i = b; i < e; ++i) ++start[(uint32_t)(pairs[i] >> 32) - lo + 1];
        for (uint32_t j = 0; j < w; ++j) start[j + 1] += start[j];
        std::vector<uint64_t> cur(start.begin(), start.end() - 1);
        std::vector<uint32_t> col(e - b);
        for (uint64_t i = b; i < e; ++i) col[cur[(uint32_t)(pairs[i] >> 32) - lo]++] = (uint32_t)pairs[i];
        // sorted, unique neighbours written back over the partition's pairs as u32
        uint32_t* dst = reinterpret_cast<uint32_t*>(pairs.data() + b);
        for (uint32_t j = 0; j < w; ++j) {
            uint32_t* cb = col.data() + start[j];
            uint32_t* ce = col.data() + start[j + 1];
            std::sort(cb, ce);
            const uint32_t k = (uint32_t)(std::unique(cb, ce) - cb);
            deg[lo + j] = k;
            std::memcpy(dst, cb, 4ull * k);
            dst += k;
        }
    }
    uint64_t nnz = 0;
    for (uint32_t j = 0; j < n; ++j) nnz += deg[j];
    if (nnz > 0xFFFFFFFFull) throw Error(BLEST_ERR_UNSUPPORTED, "more than 2^32-1 non-zeros");
    Csc g;
    g.n = n;
    g.nnz = (uint32_t)nnz;
    g.col_ptrs.assign((size_t)n + 1, 0);
    for (uint32_t j = 0; j < n; ++j) g.col_ptrs[j + 1] = g.col_ptrs[j] + deg[j];
    g.rows.resize(nnz);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t pp = 0; pp < (int64_t)P; ++pp) {
        const uint32_t p = (uint32_t)pp;
        const uint32_t lo = p << shift, hi = (uint32_t)std::min<uint64_t>(n, ((uint64_t)p + 1) << shift);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(pairs.data() + pbase[p]);
        std::memcpy(g.rows.data() + g.col_ptrs[lo], src, 4ull * (g.col_ptrs[hi] - g.col_ptrs[lo]));
    }
    g.is_social = classify_social(g);
    return g;
}

Csc csc_from_arrays(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows) {
    if (col_ptrs[0] != 0) throw Error(BLEST_ERR_INVALID_ARG, "col_ptrs[0] must be 0");
    for (uint32_t j = 0; j < n; ++j)
        if (col_ptrs[j] > col_ptrs[j + 1]) throw Error(BLEST_ERR_INVALID_ARG, "col_ptrs must be non-decreasing");
    Csc g;
    g.n = n;
    g.nnz = col_ptrs[n];
    g.col_ptrs.assign(col_ptrs, col_ptrs + n + 1);
    g.rows.assign(rows, rows + g.nnz);
    for (uint32_t p = 0; p < g.nnz; ++p)
        if (g.rows[p] >= n) throw Error(BLEST_ERR_INVALID_ARG, "row index out of range");
    sort_columns(g);
    g.is_social = classify_social(g);
    return g;
}

std::vector<uint32_t> seeded_permutation(uint32_t n, uint64_t seed) {
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; ++i) perm[i] = i;
    SeqRng rng(seed ^ 0x5EEDBEEFCAFEF00Dull);
    for (uint32_t i = n; i > 1; --i) {
        const uint32_t j = (uint32_t)rng.below(i);
        std::swap(perm[i - 1], perm[j]);
    }
    return perm;
}

std::vector<uint32_t> sample_sources(const Csc& g, uint32_t k, uint64_t seed) {
    std::vector<uint32_t> cand;
    for (uint32_t v = 0; v < g.n; ++v)
        if (g.degree(v) >= 1) cand.push_back(v);
    SeqRng rng(seed ^ 0x50C5A3B1E5ull);
    const uint32_t take = std::min<uint32_t>(k, (uint32_t)cand.size());
    for (uint32_t i = 0; i < take; ++i) {
        const uint32_t j = i + (uint32_t)rng.below(cand.size() - i);
        std::swap(cand[i], cand[j]);
    }
    cand.resize(take);
    return cand;
}

}  // namespace blest
