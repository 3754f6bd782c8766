// C ABI for the host layer (CSC, orderings, BVSS). See include/blest.h.
#include <omp.h>

#include <cstring>
#include <new>
#include <string>

#include "blest.h"
#include "objects.hpp"
#include "bvss.hpp"
#include "csc.hpp"
#include "errors.hpp"
#include "generators.hpp"
#include "reorder.hpp"


using blest::guarded;

extern "C" {

int blest_csc_read_mtx(const char* path, int undirected, int binary, blest_csc** out) {
    return guarded([&] {
        blest::require(path && out, "null argument");
        *out = new blest_csc{blest::csc_read_mtx(path, undirected != 0, binary != 0)};
    });
}

int blest_csc_read_mtx_auto(const char* path, blest_csc** out) {
    return guarded([&] {
        blest::require(path && out, "null argument");
        *out = new blest_csc{blest::csc_read_mtx_auto(path)};
    });
}

int blest_csc_load_bin(const char* path, blest_csc** out) {
    return guarded([&] {
        blest::require(path && out, "null argument");
        *out = new blest_csc{blest::csc_load_bin(path)};
    });
}

int blest_csc_save_bin(const blest_csc* g, const char* path) {
    return guarded([&] {
        blest::require(g && path, "null argument");
        blest::csc_save_bin(g->g, path);
    });
}

int blest_csc_from_arrays(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, blest_csc** out) {
    return guarded([&] {
        blest::require(col_ptrs && out && (rows || col_ptrs[n] == 0), "null argument");
        *out = new blest_csc{blest::csc_from_arrays(n, col_ptrs, rows)};
    });
}

int blest_csc_generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                            uint64_t permute_seed, blest_csc** out) {
    return guarded([&] {
        blest::require(out, "null argument");
        *out = new blest_csc{blest::generate_rmat(scale, edge_factor, a, b, c, seed, permute_seed)};
    });
}

int blest_csc_generate_grid(uint32_t width, uint32_t height, double p_delete, double shortcut_fraction,
                            uint64_t seed, uint64_t permute_seed, blest_csc** out) {
    return guarded([&] {
        blest::require(out, "null argument");
        *out = new blest_csc{blest::generate_grid(width, height, p_delete, shortcut_fraction, seed, permute_seed)};
    });
}

int blest_csc_generate_er(uint32_t n, uint64_t m, uint64_t seed, uint64_t permute_seed, blest_csc** out) {
    return guarded([&] {
        blest::require(out, "null argument");
        *out = new blest_csc{blest::generate_er(n, m, seed, permute_seed)};
    });
}

int blest_csc_view_get(const blest_csc* g, blest_csc_view* out) {
    return guarded([&] {
        blest::require(g && out, "null argument");
        out->n = g->g.n;
        out->nnz = g->g.nnz;
        out->is_social = g->g.is_social ? 1 : 0;
        out->col_ptrs = g->g.col_ptrs.data();
        out->rows = g->g.rows.data();
    });
}

int blest_csc_destroy(blest_csc* g) {
    delete g;
    return BLEST_OK;
}

int blest_csc_transpose(const blest_csc* g, blest_csc** out) {
    return guarded([&] {
        blest::require(g && out, "null argument");
        *out = new blest_csc{blest::csc_transpose(g->g)};
    });
}

int blest_csc_check_symmetry(const blest_csc* g, int* symmetric) {
    return guarded([&] {
        blest::require(g && symmetric, "null argument");
        *symmetric = blest::csc_check_symmetry(g->g) ? 1 : 0;
    });
}

int blest_csc_symmetrize(const blest_csc* g, blest_csc** out) {
    return guarded([&] {
        blest::require(g && out, "null argument");
        *out = new blest_csc{blest::csc_symmetrize(g->g)};
    });
}

int blest_csc_sample_sources(const blest_csc* g, uint32_t k, uint64_t seed, uint32_t* out, uint32_t* count) {
    return guarded([&] {
        blest::require(g && out && count, "null argument");
        const std::vector<uint32_t> s = blest::sample_sources(g->g, k, seed);
        std::memcpy(out, s.data(), 4ull * s.size());
        *count = (uint32_t)s.size();
    });
}

int blest_csc_reorder(blest_csc* g, const blest_order_params* p, uint32_t* inverse_permutation) {
    return guarded([&] {
        blest::require(g && p && inverse_permutation, "null argument");
        int mode = p->mode;
        if (mode == BLEST_ORDER_AUTO) {
            // CSC::reorder, CSC.cuh:358-386.
            if (g->g.is_social) mode = p->jaccard_enabled ? BLEST_ORDER_JACCARD : BLEST_ORDER_NATURAL;
            else mode = BLEST_ORDER_RCM;
        }
        std::vector<uint32_t> inv;
        switch (mode) {
            case BLEST_ORDER_NATURAL: inv = blest::order_natural(g->g); break;
            case BLEST_ORDER_JACCARD:
                inv = blest::order_jaccard_window(g->g, blest::kSliceSize, p->window, p->threads);
                break;
            case BLEST_ORDER_RCM: inv = blest::order_rcm(g->g, p->rcm_rand_seed ? p->rcm_rand_seed : 1u); break;
            case BLEST_ORDER_RANDOM: inv = blest::order_random(g->g, p->seed); break;
            case BLEST_ORDER_DEGREE: inv = blest::order_degree(g->g, true); break;
            case BLEST_ORDER_GORDER:
                // CSC::gorder(sliceSize): the greedy's window is the slice size
                inv = blest::order_gorder(g->g, blest::kSliceSize);
                break;
            default: throw blest::Error(BLEST_ERR_INVALID_ARG, "unknown ordering mode");
        }
        blest::csc_apply_permutation(g->g, inv);
        std::memcpy(inverse_permutation, inv.data(), 4ull * inv.size());
    });
}

int blest_csc_apply_permutation(blest_csc* g, const uint32_t* inverse_permutation) {
    return guarded([&] {
        blest::require(g && inverse_permutation, "null argument");
        std::vector<uint32_t> inv(inverse_permutation, inverse_permutation + g->g.n);
        blest::csc_apply_permutation(g->g, inv);
    });
}

int blest_ordering_save_bin(const char* path, const uint32_t* inverse_permutation, uint32_t n) {
    return guarded([&] {
        blest::require(path && inverse_permutation, "null argument");
        blest::ordering_save_bin(std::vector<uint32_t>(inverse_permutation, inverse_permutation + n), path);
    });
}

int blest_ordering_load_bin(const char* path, uint32_t n, uint32_t* inverse_permutation) {
    return guarded([&] {
        blest::require(path && inverse_permutation, "null argument");
        const std::vector<uint32_t> inv = blest::ordering_load_bin(path, n);
        std::memcpy(inverse_permutation, inv.data(), 4ull * n);
    });
}

int blest_bvss_build(const blest_csc* g, int full_padding, blest_bvss** out) {
    return guarded([&] {
        blest::require(g && out, "null argument");
        const bool fp = full_padding < 0 ? !g->g.is_social : full_padding != 0;
        *out = new blest_bvss{blest::bvss_build(g->g, fp)};
    });
}

int blest_bvss_from_view(const blest_bvss_view* v, blest_bvss** out) {
    return guarded([&] {
        blest::require(v && out, "null argument");
        blest::require(v->slice_set_ptrs && v->real_ptrs && (v->no_virtual_slice_sets == 0 || v->virtual_to_real) &&
                           (v->no_slices == 0 || (v->row_ids && v->masks)),
                       "null array in BVSS view");
        blest::Bvss b;
        b.n = v->n;
        b.slice_size = v->slice_size;
        b.no_masks = v->no_masks;
        b.no_real = v->no_real_slice_sets;
        b.no_virtual = v->no_virtual_slice_sets;
        b.no_slices = v->no_slices;
        b.update_divergence = v->update_divergence;
        b.full_padding = v->full_padding != 0;
        b.slice_set_ptrs.assign(v->slice_set_ptrs, v->slice_set_ptrs + b.no_virtual + 1);
        b.virtual_to_real.assign(v->virtual_to_real, v->virtual_to_real + b.no_virtual);
        b.real_ptrs.assign(v->real_ptrs, v->real_ptrs + b.no_real + 1);
        b.row_ids.assign(v->row_ids, v->row_ids + b.no_slices);
        b.masks.assign(v->masks, v->masks + b.no_slices / blest::kNoMasks);
        blest::bvss_validate(b);
        uint64_t padded = 0;
        for (uint32_t w : b.masks)
            for (uint32_t k = 0; k < 4; ++k) padded += ((w >> (8 * k)) & 0xFF) == 0;
        b.no_padded = padded;
        *out = new blest_bvss{std::move(b)};
    });
}

int blest_bvss_view_get(const blest_bvss* b, blest_bvss_view* out) {
    return guarded([&] {
        blest::require(b && out, "null argument");
        const blest::Bvss& x = b->b;
        out->n = x.n;
        out->slice_size = x.slice_size;
        out->no_masks = x.no_masks;
        out->no_real_slice_sets = x.no_real;
        out->no_virtual_slice_sets = x.no_virtual;
        out->no_slices = x.no_slices;
        out->no_padded_slices = x.no_padded;
        out->update_divergence = x.update_divergence;
        out->full_padding = x.full_padding ? 1 : 0;
        out->slice_set_ptrs = x.slice_set_ptrs.data();
        out->virtual_to_real = x.virtual_to_real.data();
        out->real_ptrs = x.real_ptrs.data();
        out->row_ids = x.row_ids.data();
        out->masks = x.masks.data();
    });
}

int blest_bvss_save_bin(const blest_bvss* b, const char* path) {
    return guarded([&] {
        blest::require(b && path, "null argument");
        blest::bvss_save_bin(b->b, path);
    });
}

int blest_bvss_load_bin(const char* path, blest_bvss** out) {
    return guarded([&] {
        blest::require(path && out, "null argument");
        *out = new blest_bvss{blest::bvss_load_bin(path)};
    });
}

int blest_bvss_destroy(blest_bvss* b) {
    delete b;
    return BLEST_OK;
}

int blest_bvss_edge_check(const blest_bvss* b, uint64_t* edges) {
    return guarded([&] {
        blest::require(b && edges, "null argument");
        *edges = b->b.edge_check();
    });
}

int blest_cc_relabel_dense(const uint32_t* labels, uint32_t n, uint32_t* dense_out, uint32_t* no_components) {
    return guarded([&] {
        blest::require(labels && dense_out, "null argument");
        // Dense ids in increasing order of the label value, i.e. of the
        // component's minimum vertex id (CC/BVSSCCKernel.cuh:1268-1290).
        std::vector<uint32_t> rank(n, 0xFFFFFFFFu);
        for (uint32_t v = 0; v < n; ++v) {
            blest::require(labels[v] < n, "label out of range");
            rank[labels[v]] = 0;
        }
        uint32_t id = 0;
        for (uint32_t v = 0; v < n; ++v)
            if (rank[v] == 0) rank[v] = id++;
        for (uint32_t v = 0; v < n; ++v) dense_out[v] = rank[labels[v]];
        if (no_components) *no_components = id;
    });
}

}  // extern "C"
