// C-ABI entry points for the per-stage seams (device pointers in, device or
// host results out). Declarations and reference citations: include/p3g.h.
#pragma once
#include "context.cuh"

struct p3g_ctx {
    p3g::Ctx c;
};
struct p3g_tree {
    p3g::Tree t;
};

#define P3G_API extern "C" __attribute__((visibility("default")))

#define P3G_TRY(ctxp, ...)                                    \
    try {                                                     \
        if (ctxp) ::p3g::bind_p2((ctxp)->c);                  \
        __VA_ARGS__;                                          \
        return p3g::OK;                                       \
    } catch (const p3g::CudaError &e) {                       \
        if (ctxp) (ctxp)->c.last_error = e.what;              \
        return e.status;                                      \
    } catch (const std::bad_alloc &) {                        \
        if (ctxp) (ctxp)->c.last_error = "host allocation failed"; \
        return p3g::ERR_OOM;                                  \
    }

P3G_API int p3g_ctx_create(int device, const uint64_t *poseidon2_params130, p3g_ctx **out) {
    if (!out || !poseidon2_params130) return p3g::ERR_INVALID;
    *out = nullptr;
    p3g_ctx *x = nullptr;
    try {
        x = new p3g_ctx();
        x->c.device = device;
        CK(cudaSetDevice(device));
        CK(cudaStreamCreateWithFlags(&x->c.stream, cudaStreamNonBlocking));
        memcpy(x->c.p2, poseidon2_params130, sizeof(x->c.p2));
        p3g::bind_p2(x->c);
        x->c.make_pool();
        x->c.enable_cache(8ull << 30);  // up to 64 GB of large buffers kept between proofs
    } catch (const p3g::CudaError &e) {
        delete x;
        return e.status;
    }
    *out = x;
    return p3g::OK;
}

P3G_API void p3g_ctx_destroy(p3g_ctx *x) {
    if (!x) return;
    cudaSetDevice(x->c.device);
    // every stream-ordered buffer the context owns is freed before its streams
    x->c.release();
    delete x;
}

P3G_API const char *p3g_last_error(const p3g_ctx *x) { return x ? x->c.last_error.c_str() : "null context"; }

P3G_API int p3g_coset_lde(p3g_ctx *x, const uint64_t *d_in, uint64_t height, uint64_t width, uint32_t log_blowup,
                          uint64_t shift, uint64_t *d_out) {
    if (!x || !d_in || !d_out || height == 0 || (height & (height - 1)) || log_blowup > 8) return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        p3g::DBuf tmp = x->c.alloc(height * width);
        p3g::coset_lde(x->c, d_in, width, height, width, log_blowup, shift % gl::P, d_out, tmp.p);
        x->c.sync();
    })
}

// PeriodicLde::build (p3-miden-lifted-stark/src/prover/periodic.rs:49-81):
// the periodic columns repeated to the largest period (max_period x width,
// row-major, on the device) extended on the coset of shift
// lde_shift^(trace_height / max_period), natural order. d_out holds
// (max_period << log_blowup) x width; the constraint evaluation reads row
// i mod that height (periodic.rs:88-98).
P3G_API int p3g_periodic_lde(p3g_ctx *x, const uint64_t *d_repeated, uint64_t max_period, uint64_t width,
                             uint32_t log_blowup, uint32_t log_trace_height, uint64_t lde_shift, uint64_t *d_out) {
    if (!x || !d_repeated || !d_out || max_period == 0 || (max_period & (max_period - 1)) || log_blowup > 8 ||
        log_trace_height > 32 || max_period > (1ull << log_trace_height) || width == 0)
        return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        const uint32_t log_p = p3g::log2u(max_period), L = log_p + log_blowup;
        const uint64_t shift = gl::exp2k(lde_shift % gl::P, log_trace_height - log_p);
        p3g::DBuf tmp = x->c.alloc(max_period * width), brev = x->c.alloc((max_period << log_blowup) * width);
        p3g::coset_lde(x->c, d_repeated, width, max_period, width, log_blowup, shift, brev.p, tmp.p);
        const uint64_t n = (max_period << log_blowup) * width;
        p3g::bitrev_rows_kernel<<<(unsigned)((n + 255) / 256), 256, 0, x->c.stream>>>(brev.p, d_out, L, width);
        CK(cudaGetLastError());
        x->c.launches++;
        x->c.sync();
    })
}

P3G_API int p3g_lmcs_build(p3g_ctx *x, const uint64_t *const *d_mats, const uint64_t *heights, const uint64_t *widths,
                           uint64_t n, uint32_t alignment, p3g_tree **out) {
    if (!x || !d_mats || !heights || !widths || !out || n == 0 || n > 64) return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n; i++) {
        if (heights[i] == 0 || (heights[i] & (heights[i] - 1))) return p3g::ERR_INVALID;
        if (i && heights[i] < heights[i - 1]) return p3g::ERR_VALIDATION;
    }
    *out = nullptr;
    p3g_tree *t = new p3g_tree();
    try {
        CK(cudaSetDevice(x->c.device));
        p3g::bind_p2(x->c);
        std::vector<p3g::Mat> mats;
        for (uint64_t i = 0; i < n; i++) mats.push_back({d_mats[i], heights[i], widths[i]});
        p3g::build_tree(x->c, t->t, mats, alignment);
        x->c.sync();
    } catch (const p3g::CudaError &e) {
        x->c.last_error = e.what;
        delete t;
        return e.status;
    }
    *out = t;
    return p3g::OK;
}

// HidingLmcsConfig::build_tree / build_aligned_tree
// (p3-miden-lmcs/src/hiding_lmcs.rs:112-145) with the caller's salt matrix
// (tree height x salt_width, row-major, on the device; borrowed like the
// matrices).
P3G_API int p3g_lmcs_build_hiding(p3g_ctx *x, const uint64_t *const *d_mats, const uint64_t *heights,
                                  const uint64_t *widths, uint64_t n, uint32_t alignment, const uint64_t *d_salt,
                                  uint64_t salt_width, p3g_tree **out) {
    if (!x || !d_mats || !heights || !widths || !out || !d_salt || n == 0 || n > 64) return p3g::ERR_INVALID;
    if (salt_width == 0 || salt_width > 4096) return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n; i++) {
        if (heights[i] == 0 || (heights[i] & (heights[i] - 1))) return p3g::ERR_INVALID;
        if (i && heights[i] < heights[i - 1]) return p3g::ERR_VALIDATION;
    }
    *out = nullptr;
    p3g_tree *t = new p3g_tree();
    try {
        CK(cudaSetDevice(x->c.device));
        p3g::bind_p2(x->c);
        std::vector<p3g::Mat> mats;
        for (uint64_t i = 0; i < n; i++) mats.push_back({d_mats[i], heights[i], widths[i]});
        const p3g::Mat salt{d_salt, heights[n - 1], salt_width};
        p3g::build_tree(x->c, t->t, mats, alignment, &salt);
        x->c.sync();
    } catch (const p3g::CudaError &e) {
        x->c.last_error = e.what;
        delete t;
        return e.status;
    }
    *out = t;
    return p3g::OK;
}

P3G_API int p3g_lmcs_root(const p3g_tree *t, uint64_t *out4) {
    if (!t || !out4) return p3g::ERR_INVALID;
    memcpy(out4, t->t.root, 32);
    return p3g::OK;
}

P3G_API int p3g_lmcs_layer(p3g_ctx *x, const p3g_tree *t, uint32_t level, uint64_t *host_out) {
    if (!x || !t || !host_out || level > t->t.depth) return p3g::ERR_INVALID;
    P3G_TRY(x, {
        uint64_t n = t->t.H >> level;
        CK(cudaMemcpyAsync(host_out, t->t.layers.p + 4 * t->t.layer_off(level), n * 32, cudaMemcpyDeviceToHost,
                           x->c.stream));
        x->c.sync();
    })
}

P3G_API void p3g_lmcs_free(p3g_tree *t) { delete t; }

namespace p3g {
__global__ void permute_batch_kernel(uint64_t *st, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t s[12];
#pragma unroll
    for (int k = 0; k < 12; k++) s[k] = st[i * 12 + k];
    p2_permute_dev(s);
#pragma unroll
    for (int k = 0; k < 12; k++) st[i * 12 + k] = p2w::canon(s[k]);
}
}  // namespace p3g

P3G_API int p3g_poseidon2_permute_batch(p3g_ctx *x, uint64_t *d_states, uint64_t n) {
    if (!x || (!d_states && n)) return p3g::ERR_INVALID;
    P3G_TRY(x, {
        if (n) {
            p3g::permute_batch_kernel<<<(unsigned)((n + 127) / 128), 128, 0, x->c.stream>>>(d_states, n);
            CK(cudaGetLastError());
        }
        x->c.sync();
    })
}

#include "host_rng.cuh"

// Poseidon2Goldilocks<12> constants as the goldilocks_poseidon2 dev config
// builds them (SmallRng::seed_from_u64(2025)), with the placeholder diagonal.
P3G_API void p3g_default_poseidon2_params(uint64_t *out130) {
    uint64_t diag[12];
    p3g::placeholder_diag(diag);
    p3g::poseidon2_params_from_seed(2025, diag, out130);
}
P3G_API void p3g_poseidon2_params_from_seed(uint64_t seed, const uint64_t *diag12, uint64_t *out130) {
    p3g::poseidon2_params_from_seed(seed, diag12, out130);
}
