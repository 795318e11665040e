// C ABI of the host symbolic phase (see include/cliqgpu.h).
#include <new>

#include "cliqgpu_internal.h"

struct cliq_symbolic_s {
    cliqgpu::Symbolic s;
};

using cliqgpu::Symbolic;

extern "C" {

int cliq_natural_nested_dissection(int32_t nx, int32_t ny, int32_t nz, int64_t n, const int64_t* rowptr,
                                   const int32_t* colind, int32_t cutoff, cliq_symbolic* out) {
    if (!out) return CLIQ_ERR_ARG;
    *out = nullptr;
    cliq_symbolic h = new (std::nothrow) cliq_symbolic_s;
    if (!h) return CLIQ_ERR_OOM;
    int st;
    try {
        st = cliqgpu::natural_nested_dissection(nx, ny, nz, n, rowptr, colind, cutoff, h->s);
    } catch (const std::bad_alloc&) {
        st = CLIQ_ERR_OOM;
    }
    if (st != CLIQ_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CLIQ_OK;
}

int cliq_nested_dissection(int64_t n, const int64_t* rowptr, const int32_t* colind, int32_t cutoff, int32_t num_seps,
                           cliq_symbolic* out) {
    if (!out) return CLIQ_ERR_ARG;
    *out = nullptr;
    cliq_symbolic h = new (std::nothrow) cliq_symbolic_s;
    if (!h) return CLIQ_ERR_OOM;
    int st;
    try {
        st = cliqgpu::graph_nested_dissection(n, rowptr, colind, cutoff, num_seps, h->s);
    } catch (const std::bad_alloc&) {
        st = CLIQ_ERR_OOM;
    }
    if (st != CLIQ_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CLIQ_OK;
}

int cliq_batch_nested_dissection(int32_t count, const int32_t* dims, int64_t n, const int64_t* rowptr,
                                 const int32_t* colind, int32_t cutoff, cliq_symbolic* out) {
    if (!out) return CLIQ_ERR_ARG;
    *out = nullptr;
    cliq_symbolic h = new (std::nothrow) cliq_symbolic_s;
    if (!h) return CLIQ_ERR_OOM;
    int st;
    try {
        st = cliqgpu::batch_nested_dissection(count, dims, n, rowptr, colind, cutoff, h->s);
    } catch (const std::bad_alloc&) {
        st = CLIQ_ERR_OOM;
    }
    if (st != CLIQ_OK) {
        delete h;
        return st;
    }
    *out = h;
    return CLIQ_OK;
}

int cliq_symbolic_info(cliq_symbolic h, cliq_symm_info* out) {
    if (!h || !out) return CLIQ_ERR_ARG;
    Symbolic& S = h->s;
    out->num_nodes = S.num_nodes;
    out->size = S.size.data();
    out->off = S.off.data();
    out->parent = S.parent.data();
    out->children = S.children.data();
    out->lower_ptr = S.lower_ptr.data();
    out->lower = S.lower_flat.data();
    out->orig_lower_ptr = S.orig_ptr.data();
    out->orig_lower = S.orig_flat.data();
    return CLIQ_OK;
}

int cliq_symbolic_node(cliq_symbolic h, int32_t s, int32_t out[10]) {
    if (!h || !out || s < 0 || s >= h->s.num_nodes) return CLIQ_ERR_ARG;
    const Symbolic& S = h->s;
    out[0] = S.size[s];
    out[1] = S.off[s];
    out[2] = S.my_off[s];
    out[3] = S.parent[s];
    out[4] = S.children[2 * s];
    out[5] = S.children[2 * s + 1];
    out[6] = S.on_left[s];
    out[7] = (int32_t)S.lower[s].size();
    out[8] = (int32_t)S.orig_lower[s].size();
    out[9] = S.sep_parent[s];
    return CLIQ_OK;
}

int cliq_symbolic_node_array(cliq_symbolic h, int32_t s, int32_t which, int32_t* out, int64_t* len) {
    if (!h || s < 0 || s >= h->s.num_nodes || !len) return CLIQ_ERR_ARG;
    const Symbolic& S = h->s;
    const std::vector<int>* v = nullptr;
    switch (which) {
        case 0: v = &S.lower[s]; break;
        case 1: v = &S.orig_lower[s]; break;
        case 2: v = &S.orig_rel[s]; break;
        case 3: v = &S.left_rel[s]; break;
        case 4: v = &S.right_rel[s]; break;
        case 5: v = &S.inds[s]; break;
        default: return CLIQ_ERR_ARG;
    }
    *len = (int64_t)v->size();
    if (out)
        for (size_t i = 0; i < v->size(); ++i) out[i] = (*v)[i];
    return CLIQ_OK;
}

int cliq_symbolic_map(cliq_symbolic h, int32_t* map, int32_t* inverse_map) {
    if (!h) return CLIQ_ERR_ARG;
    const Symbolic& S = h->s;
    for (int64_t i = 0; i < S.n; ++i) {
        if (map) map[i] = S.map[i];
        if (inverse_map) inverse_map[i] = S.inv_map[i];
    }
    return CLIQ_OK;
}

void cliq_symbolic_destroy(cliq_symbolic h) { delete h; }

}  // extern "C"
