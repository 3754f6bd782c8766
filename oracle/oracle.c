/*
 * oracle.c -- CPU oracle for the BLEST B200 hot path (test infrastructure;
 * see oracle.h). Plain C99 + OpenMP.
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

int oracle_bfs_csc(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t src, uint32_t* levels) {
    if (src >= n) return 1;
    uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    if (!q) return 2;
    for (uint32_t v = 0; v < n; ++v) levels[v] = ORACLE_UNREACHED;
    uint32_t head = 0, tail = 0;
    levels[src] = 0;
    q[tail++] = src;
    while (head < tail) {
        const uint32_t u = q[head++];
        for (uint32_t p = col_ptrs[u]; p < col_ptrs[u + 1]; ++p) {
            const uint32_t v = rows[p];
            if (levels[v] == ORACLE_UNREACHED) {
                levels[v] = levels[u] + 1;
                q[tail++] = v;
            }
        }
    }
    free(q);
    return 0;
}

int oracle_bfs_bvss(uint32_t n, uint32_t no_real, const uint64_t* ssp, const uint32_t* real_ptrs,
                    const uint32_t* row_ids, const uint32_t* masks, uint32_t src, uint32_t* levels) {
    if (src >= n) return 1;
    const uint32_t words = (n + 31) / 32;
    uint32_t* frontier = (uint32_t*)calloc(words + 1, 4);
    uint32_t* next = (uint32_t*)calloc(words + 1, 4);
    if (!frontier || !next) return 2;
    for (uint32_t v = 0; v < n; ++v) levels[v] = ORACLE_UNREACHED;
    levels[src] = 0;
    frontier[src >> 5] = 1u << (src & 31);
    const uint8_t* fbytes = (const uint8_t*)frontier;
    for (uint32_t level = 1;; ++level) {
        int any = 0;
        memset(next, 0, 4 * (size_t)words);
        for (uint32_t r = 0; r < no_real; ++r) {
            const uint32_t fb = fbytes[r];
            if (!fb) continue;
            for (uint32_t v = real_ptrs[r]; v < real_ptrs[r + 1]; ++v) {
                for (uint64_t s = ssp[v]; s < ssp[v + 1]; ++s) {
                    const uint32_t mb = (masks[s >> 2] >> (8 * (s & 3))) & 0xFFu;
                    if (!(mb & fb)) continue;
                    const uint32_t row = row_ids[s];
                    if (row >= n) return 3; /* hit on a padding slice */
                    if (levels[row] == ORACLE_UNREACHED) {
                        levels[row] = level;
                        next[row >> 5] |= 1u << (row & 31);
                        any = 1;
                    }
                }
            }
        }
        if (!any) break;
        uint32_t* t = frontier;
        frontier = next;
        next = t;
        fbytes = (const uint8_t*)frontier;
    }
    free(frontier);
    free(next);
    return 0;
}

int oracle_cc_csc(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t* labels) {
    uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint8_t* inq = (uint8_t*)calloc(n ? n : 1, 1);
    if (!q || !inq) return 2;
    for (uint32_t v = 0; v < n; ++v) labels[v] = v;
    /* Visit sources in increasing id: a BFS from u labels every vertex it
     * reaches that has no smaller label yet; the first source to reach v
     * is the smallest id reaching v, so each vertex is labelled once. */
    uint8_t* done = (uint8_t*)calloc(n ? n : 1, 1);
    if (!done) return 2;
    for (uint32_t u = 0; u < n; ++u) {
        if (done[u]) continue;
        uint32_t head = 0, tail = 0;
        q[tail++] = u;
        done[u] = 1;
        while (head < tail) {
            const uint32_t x = q[head++];
            for (uint32_t p = col_ptrs[x]; p < col_ptrs[x + 1]; ++p) {
                const uint32_t y = rows[p];
                if (!done[y]) {
                    done[y] = 1;
                    labels[y] = u;
                    q[tail++] = y;
                }
            }
        }
    }
    free(q);
    free(inq);
    free(done);
    return 0;
}

int oracle_cc_bvss(uint32_t n, uint32_t no_real, const uint64_t* ssp, const uint32_t* real_ptrs,
                   const uint32_t* row_ids, const uint32_t* masks, uint32_t* labels) {
    const uint32_t words = (n + 31) / 32;
    uint32_t* active = (uint32_t*)calloc(words + 1, 4);
    uint32_t* next = (uint32_t*)calloc(words + 1, 4);
    uint32_t* old = (uint32_t*)malloc(4 * (size_t)(n ? n : 1));
    if (!active || !next || !old) return 2;
    for (uint32_t v = 0; v < n; ++v) {
        labels[v] = v;
        active[v >> 5] |= 1u << (v & 31);
    }
    for (;;) {
        int changed = 0;
        memcpy(old, labels, 4 * (size_t)n);
        memset(next, 0, 4 * (size_t)words);
        const uint8_t* ab = (const uint8_t*)active;
        for (uint32_t r = 0; r < no_real; ++r) {
            const uint32_t fb = ab[r];
            if (!fb) continue;
            for (uint32_t v = real_ptrs[r]; v < real_ptrs[r + 1]; ++v) {
                for (uint64_t s = ssp[v]; s < ssp[v + 1]; ++s) {
                    uint32_t hit = ((masks[s >> 2] >> (8 * (s & 3))) & 0xFFu) & fb;
                    if (!hit) continue;
                    const uint32_t row = row_ids[s];
                    if (row >= n) return 3;
                    uint32_t m = labels[row];
                    while (hit) {
                        const uint32_t col = r * 8 + (uint32_t)__builtin_ctz(hit);
                        if (old[col] < m) m = old[col];
                        hit &= hit - 1;
                    }
                    if (m < labels[row]) {
                        labels[row] = m;
                        next[row >> 5] |= 1u << (row & 31);
                        changed = 1;
                    }
                }
            }
        }
        if (!changed) break;
        uint32_t* t = active;
        active = next;
        next = t;
    }
    free(active);
    free(next);
    free(old);
    return 0;
}

int64_t oracle_check_parents(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t src,
                             const uint32_t* levels, const uint32_t* parents) {
    if (src >= n || parents[src] != src || levels[src] != 0) return 1 + (int64_t)src;
    for (uint32_t v = 0; v < n; ++v) {
        if (v == src) continue;
        if (levels[v] == ORACLE_UNREACHED) {
            if (parents[v] != ORACLE_UNREACHED) return 1 + (int64_t)v;
            continue;
        }
        const uint32_t p = parents[v];
        if (p >= n || levels[p] == ORACLE_UNREACHED || levels[p] + 1 != levels[v]) return 1 + (int64_t)v;
        /* edge p -> v: v among the rows of column p (sorted) */
        uint32_t lo = col_ptrs[p], hi = col_ptrs[p + 1];
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (rows[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        if (lo == col_ptrs[p + 1] || rows[lo] != v) return 1 + (int64_t)v;
    }
    return 0;
}

int oracle_bfs_omp(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, const uint32_t* in_ptrs,
                   const uint32_t* in_ids, uint32_t src, uint32_t* levels, int threads) {
    if (src >= n) return -1;
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    const uint32_t words = (n + 63) / 64;
    uint64_t* front = (uint64_t*)calloc(words + 1, 8);
    uint64_t* nextb = (uint64_t*)calloc(words + 1, 8);
    uint32_t* queue = (uint32_t*)malloc(4 * (size_t)(n ? n : 1));
    uint32_t* nqueue = (uint32_t*)malloc(4 * (size_t)(n ? n : 1));
    if (!front || !nextb || !queue || !nqueue) return -2;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t v = 0; v < (int64_t)n; ++v) levels[v] = ORACLE_UNREACHED;
    uint64_t m_total = col_ptrs[n];
    levels[src] = 0;
    queue[0] = src;
    uint32_t qsize = 1;
    uint64_t m_f = col_ptrs[src + 1] - col_ptrs[src];
    uint64_t m_u = m_total - m_f;
    int bottom_up = 0;
    const double alpha = 14.0, beta = 24.0;
    for (uint32_t level = 1; qsize > 0; ++level) {
        if (!bottom_up && (double)m_f > (double)m_u / alpha) bottom_up = 1;
        else if (bottom_up && (double)qsize < (double)n / beta) bottom_up = 0;
        uint32_t nsize = 0;
        uint64_t nm = 0;
        if (bottom_up) {
            memset(front, 0, 8 * (size_t)words);
#pragma omp parallel for num_threads(nt) schedule(static)
            for (int64_t i = 0; i < (int64_t)qsize; ++i) {
                const uint32_t v = queue[i];
                __atomic_fetch_or(&front[v >> 6], 1ull << (v & 63), __ATOMIC_RELAXED);
            }
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024) reduction(+ : nm)
            for (int64_t v = 0; v < (int64_t)n; ++v) {
                if (levels[v] != ORACLE_UNREACHED) continue;
                for (uint32_t p = in_ptrs[v]; p < in_ptrs[v + 1]; ++p) {
                    const uint32_t u = in_ids[p];
                    if ((front[u >> 6] >> (u & 63)) & 1) {
                        levels[v] = level;
                        nm += col_ptrs[v + 1] - col_ptrs[v];
                        break;
                    }
                }
            }
            /* rebuild the queue from the new level (ordered by id) */
            uint32_t cnt = 0;
            for (uint32_t v = 0; v < n; ++v)
                if (levels[v] == level) nqueue[cnt++] = v;
            nsize = cnt;
        } else {
#pragma omp parallel num_threads(nt) reduction(+ : nm)
            {
#pragma omp for schedule(dynamic, 64)
                for (int64_t i = 0; i < (int64_t)qsize; ++i) {
                    const uint32_t u = queue[i];
                    for (uint32_t p = col_ptrs[u]; p < col_ptrs[u + 1]; ++p) {
                        const uint32_t v = rows[p];
                        if (__atomic_load_n(&levels[v], __ATOMIC_RELAXED) != ORACLE_UNREACHED) continue;
                        uint32_t expect = ORACLE_UNREACHED;
                        if (__atomic_compare_exchange_n(&levels[v], &expect, level, 0, __ATOMIC_RELAXED,
                                                        __ATOMIC_RELAXED)) {
                            const uint32_t pos = __atomic_fetch_add(&nsize, 1u, __ATOMIC_RELAXED);
                            nqueue[pos] = v;
                            nm += col_ptrs[v + 1] - col_ptrs[v];
                        }
                    }
                }
            }
        }
        uint32_t* t = queue;
        queue = nqueue;
        nqueue = t;
        qsize = nsize;
        m_f = nm;
        m_u -= nm;
    }
    free(front);
    free(nextb);
    free(queue);
    free(nqueue);
    return nt;
}

int oracle_cc_omp(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t* labels, int threads) {
    const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nt)
    for (int64_t v = 0; v < (int64_t)n; ++v) labels[v] = (uint32_t)v;
    int changed = 1;
    while (changed) {
        changed = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1024) reduction(| : changed)
        for (int64_t u = 0; u < (int64_t)n; ++u) {
            const uint32_t lu = __atomic_load_n(&labels[u], __ATOMIC_RELAXED);
            for (uint32_t p = col_ptrs[u]; p < col_ptrs[u + 1]; ++p) {
                const uint32_t v = rows[p];
                uint32_t lv = __atomic_load_n(&labels[v], __ATOMIC_RELAXED);
                while (lu < lv) {
                    if (__atomic_compare_exchange_n(&labels[v], &lv, lu, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
                        changed = 1;
                        break;
                    }
                }
            }
        }
    }
    return nt;
}

uint64_t oracle_reached_degree_sum(uint32_t n, const uint32_t* col_ptrs, const uint32_t* levels) {
    uint64_t s = 0;
    for (uint32_t v = 0; v < n; ++v)
        if (levels[v] != ORACLE_UNREACHED) s += col_ptrs[v + 1] - col_ptrs[v];
    return s;
}
