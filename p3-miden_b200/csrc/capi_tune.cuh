// Autotuning of launch shapes: the bit ranges of the coset LDE and the
// column-slab width of the main commit, timed on the context's device with
// CUDA events, and setters that load a saved choice. Every choice computes
// the same values (exact arithmetic), so tuning changes only the time.
// Declarations: include/p3g.h.
#pragma once
#include <functional>

#include "capi_prove.cuh"

namespace p3g {
// Candidate splits of L bits: the fewest ranges that fit (ceil(L / 10)) with
// every composition whose parts lie within 3 bits of the even split, and the
// even split into one more range.
inline std::vector<std::vector<uint32_t>> split_candidates(uint32_t L) {
    std::vector<std::vector<uint32_t>> out;
    if (L == 0) return out;
    const uint32_t n = (L + 9) / 10;
    std::vector<uint32_t> cur;
    std::function<void(uint32_t, uint32_t)> rec = [&](uint32_t left, uint32_t parts) {
        if (parts == 0) {
            if (left == 0) out.push_back(cur);
            return;
        }
        const uint32_t even = L / n;
        for (uint32_t k = (even > 3 ? even - 3 : 1); k <= std::min<uint32_t>(10, even + 3); k++) {
            if (k > left) break;
            cur.push_back(k);
            rec(left - k, parts - 1);
            cur.pop_back();
        }
    };
    rec(L, n);
    if (L >= 2 * (n + 1)) out.push_back(pass_sizes_n(L, n + 1));
    return out;
}
}  // namespace p3g

// Times every candidate split of a 2^log_height x width coset LDE at
// log_blowup (reps timed runs each, after one warm-up) on random data, keeps
// the fastest for this context (later LDEs of that height use it) and
// returns it in best_sizes (*n_sizes: capacity on entry, count on return)
// with its time per LDE in *best_ms and the default split's in *default_ms.
P3G_API int p3g_autotune_lde(p3g_ctx *x, uint32_t log_height, uint64_t width, uint32_t log_blowup, uint32_t reps,
                             uint32_t *best_sizes, uint32_t *n_sizes, double *best_ms, double *default_ms) {
    if (!x || !best_sizes || !n_sizes || !best_ms || !default_ms || log_height == 0 || log_height > 24 ||
        width == 0 || log_blowup > 8 || reps == 0 || reps > 100 || (width << (log_height + log_blowup)) > (1ull << 34))
        return p3g::ERR_INVALID;
    P3G_TRY(x, {
        p3g::Ctx &c = x->c;
        CK(cudaSetDevice(c.device));
        const uint64_t h = 1ull << log_height;
        std::vector<std::vector<uint32_t>> cands = p3g::split_candidates(log_height);
        const std::vector<uint32_t> def = p3g::pass_sizes(log_height);
        if (std::find(cands.begin(), cands.end(), def) == cands.end()) cands.push_back(def);
        p3g::DBuf in = c.alloc(h * width), out = c.alloc((h << log_blowup) * width), tmp = c.alloc(h * width);
        // deterministic filler, canonical words
        CK(cudaMemsetAsync(in.p, 0x17, h * width * 8, c.stream));  // 0x1717.. < p
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        auto saved = c.lde_split;
        double best = 1e30, dflt = 0;
        std::vector<uint32_t> best_split = def;
        for (const auto &cand : cands) {
            c.lde_split[log_height] = cand;
            p3g::LdePlan plan = p3g::lde_plan(c, h, log_blowup, 7);
            p3g::lde_run(c, plan, in.p, width, width, out.p, width, tmp.p, c.stream);
            CK(cudaEventRecord(e0, c.stream));
            for (uint32_t r = 0; r < reps; r++) p3g::lde_run(c, plan, in.p, width, width, out.p, width, tmp.p, c.stream);
            CK(cudaEventRecord(e1, c.stream));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            const double per = ms / reps;
            if (cand == def) dflt = per;
            if (per < best) best = per, best_split = cand;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c.lde_split = saved;
        c.lde_split[log_height] = best_split;
        if (*n_sizes < best_split.size()) throw p3g::CudaError{p3g::ERR_INVALID, "n_sizes too small"};
        for (size_t i = 0; i < best_split.size(); i++) best_sizes[i] = best_split[i];
        *n_sizes = (uint32_t)best_split.size();
        *best_ms = best;
        *default_ms = dflt;
        c.sync();
    })
}

// Times the main commit (coset LDE of every slab plus the leaf sponge and
// the tree) of a device-resident 2^log_height x width trace at log_blowup
// for slab widths of about width/16 .. width (multiples of 8, the last one
// rounded up past the width: one slab), keeps the
// fastest for this context and returns it with its time and the default's.
P3G_API int p3g_autotune_slabs(p3g_ctx *x, uint32_t log_height, uint64_t width, uint32_t log_blowup, uint32_t reps,
                               uint64_t *best_cols, double *best_ms, double *default_ms) {
    if (!x || !best_cols || !best_ms || !default_ms || log_height == 0 || log_height > 24 || width < 8 ||
        log_blowup > 8 || reps == 0 || reps > 20 || (width << (log_height + log_blowup)) > (1ull << 34))
        return p3g::ERR_INVALID;
    P3G_TRY(x, {
        p3g::Ctx &c = x->c;
        CK(cudaSetDevice(c.device));
        const uint64_t h = 1ull << log_height;
        p3g::DBuf tr = c.alloc(h * width);
        CK(cudaMemsetAsync(tr.p, 0x17, h * width * 8, c.stream));
        p3g::Instance I{p3g::AIR_CUBIC, 1, h, width, tr.p, nullptr, 0};
        std::vector<uint64_t> cands;
        for (uint64_t div : {16, 8, 4, 2, 1}) {
            // a multiple of the rate: the last slab of a trace takes what is left
            uint64_t sw = ((width + div - 1) / div + 7) / 8 * 8;
            if (std::find(cands.begin(), cands.end(), sw) == cands.end()) cands.push_back(sw);
        }
        cands.push_back(0);  // the default rule
        cudaEvent_t e0, e1, ev_lde;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventCreate(&ev_lde));
        const uint64_t saved = c.slab_cols;
        double best = 1e30, dflt = 0;
        uint64_t best_sw = 0;
        for (uint64_t sw : cands) {
            c.slab_cols = sw;
            double total = 0;
            for (uint32_t r = 0; r <= reps; r++) {
                std::vector<p3g::DBuf> lde(1);
                std::vector<p3g::Mat> mats;
                p3g::Tree t;
                p3g::ProofOut po;
                CK(cudaEventRecord(e0, c.stream));
                p3g::commit_main_pipelined(c, &I, 1, log_blowup, log_height, lde, mats, t, po, ev_lde, {nullptr});
                CK(cudaEventRecord(e1, c.stream));
                CK(cudaEventSynchronize(e1));
                float ms = 0;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (r) total += ms;  // the first run is the warm-up
            }
            const double per = total / reps;
            if (sw == 0) dflt = per;
            if (per < best) best = per, best_sw = sw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(ev_lde);
        c.slab_cols = best_sw ? best_sw : saved;
        *best_cols = best_sw;
        *best_ms = best;
        *default_ms = dflt;
        c.sync();
    })
}

// Loads a saved split for LDEs of 2^log_height rows (P3G_ERR_INVALID unless
// every range has 1..10 bits and they add up to log_height); n = 0 restores
// the default.
P3G_API int p3g_ctx_set_lde_split(p3g_ctx *x, uint32_t log_height, const uint32_t *sizes, uint32_t n) {
    if (!x || (n && !sizes)) return p3g::ERR_INVALID;
    if (n == 0) {
        x->c.lde_split.erase(log_height);
        return p3g::OK;
    }
    std::vector<uint32_t> v(sizes, sizes + n);
    if (!p3g::valid_split(log_height, v)) return p3g::ERR_INVALID;
    x->c.lde_split[log_height] = v;
    return p3g::OK;
}
// Loads a saved slab width for the main commit (a multiple of 8; 0 restores
// the default rule).
P3G_API int p3g_ctx_set_slab_columns(p3g_ctx *x, uint64_t cols) {
    if (!x || (cols % 8) != 0) return p3g::ERR_INVALID;
    x->c.slab_cols = cols;
    return p3g::OK;
}
// DAG nodes per generated constraint kernel for the symbolic AIRs this
// context creates afterwards (0 restores the default). Fewer nodes: shorter
// kernels (instruction cache) but more launches re-reading shared cells.
P3G_API int p3g_ctx_set_air_chunk_nodes(p3g_ctx *x, uint64_t nodes) {
    if (!x || (nodes && nodes < 16)) return p3g::ERR_INVALID;
    x->c.air_chunk_nodes = nodes;
    return p3g::OK;
}

// Memory statistics of the context's pool: bytes reserved from the device,
// bytes in use by live buffers, and the host time spent in allocation calls
// since the context was created (a pool that grows maps new device memory
// inside those calls).
P3G_API int p3g_ctx_memory_stats(p3g_ctx *x, uint64_t *reserved_bytes, uint64_t *used_bytes, double *alloc_ms) {
    if (!x || !reserved_bytes || !used_bytes || !alloc_ms) return p3g::ERR_INVALID;
    *reserved_bytes = *used_bytes = 0;
    if (x->c.pool) {
        uint64_t r = 0, u = 0;  // the attributes are 64-bit values
        if (cudaMemPoolGetAttribute(x->c.pool, cudaMemPoolAttrReservedMemCurrent, &r) != cudaSuccess ||
            cudaMemPoolGetAttribute(x->c.pool, cudaMemPoolAttrUsedMemCurrent, &u) != cudaSuccess)
            return p3g::ERR_CUDA;
        *reserved_bytes = r, *used_bytes = u;
    }
    *alloc_ms = x->c.alloc_ms;
    return p3g::OK;
}
