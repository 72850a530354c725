// C ABI of the verifier (verifier.cuh): verify_multi
// (p3-miden-lifted-stark/src/verifier/mod.rs:170-364) for the proofs of
// p3g_prove, with the openings, DEEP and FRI query checks on the device.
#pragma once
#include "verifier.cuh"

typedef struct {
    double host_ms;    // transcript replay and opening layout
    double device_ms;  // uploads, kernels and read-back (CUDA events)
    uint64_t gpu_launches;
} p3g_verify_stats_c;

namespace p3g {
// Arguments of one verification: pointers, PCS parameters, AIR shapes, and
// transcript words that are canonical field elements.
inline bool words_canonical(const uint64_t *w, uint64_t n) {
    uint64_t bad = 0;
    for (uint64_t i = 0; i < n; i++) bad |= w[i] >= gl::P;
    return !bad;
}
inline int verify_args_ok(const p3g_pcs_params_c *pcs, const p3g_instance_c *inst, uint64_t n, const uint64_t *fields,
                          uint64_t n_fields, const uint64_t *commits, uint64_t n_commits, const uint64_t *digest12,
                          bool scan_words = true) {
    if (!pcs || !inst || !digest12 || n == 0 || n > 8) return ERR_INVALID;
    if ((!fields && n_fields) || (!commits && n_commits)) return ERR_INVALID;
    if (pcs->log_folding_arity < 1 || pcs->log_folding_arity > 3 || pcs->log_blowup == 0 || pcs->log_blowup > 8 ||
        pcs->num_queries == 0 || pcs->folding_pow_bits > 30 || pcs->deep_pow_bits > 30 || pcs->query_pow_bits > 30)
        return ERR_INVALID;
    for (uint64_t i = 0; i < n; i++) {
        const p3g_instance_c &I = inst[i];
        if (I.height > (1ull << 30)) return ERR_INVALID;
        if (int v = validate_air(I)) return v;
    }
    if (scan_words && !(words_canonical(fields, n_fields) && words_canonical(commits, 4 * n_commits) &&
                        words_canonical(digest12, 12)))
        return ERR_INVALID;
    return OK;
}
inline std::vector<Instance> shapes_of(const p3g_instance_c *inst, uint64_t n) {
    std::vector<Instance> ins(n);
    for (uint64_t i = 0; i < n; i++)
        ins[i] = to_instance(inst[i]), ins[i].trace_on_device = 0, ins[i].trace = nullptr;
    return ins;
}
inline PcsParams pcs_of(const p3g_pcs_params_c *pcs) {
    return PcsParams{pcs->log_blowup,    pcs->log_folding_arity, pcs->log_final_degree, pcs->folding_pow_bits,
                     pcs->deep_pow_bits, pcs->num_queries,       pcs->query_pow_bits};
}
}  // namespace p3g

P3G_API int p3g_verify(p3g_ctx *x, const p3g_pcs_params_c *pcs, const p3g_instance_c *inst, uint64_t n,
                       const uint64_t *fields, uint64_t n_fields, const uint64_t *commits, uint64_t n_commits,
                       const uint64_t *digest12, int32_t *verdict, p3g_verify_stats_c *stats) {
    if (!x || !verdict) return p3g::ERR_INVALID;
    if (int e = p3g::verify_args_ok(pcs, inst, n, fields, n_fields, commits, n_commits, digest12)) return e;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        const std::vector<p3g::Instance> ins = p3g::shapes_of(inst, n);
        p3g::vfy::Timing tm;
        *verdict = p3g::vfy::verify(x->c, p3g::pcs_of(pcs), ins.data(), n, fields, n_fields, commits, n_commits,
                                    digest12, &tm);
        if (stats) *stats = p3g_verify_stats_c{tm.host_ms, tm.device_ms, tm.launches};
    })
}

typedef struct {
    p3g_pcs_params_c pcs;
    const p3g_instance_c *instances;
    uint64_t n_instances;
    const uint64_t *fields;
    uint64_t n_fields;
    const uint64_t *commits;
    uint64_t n_commits;
    const uint64_t *digest12;
} p3g_verify_job_c;

// Several proofs in one call: the host replays on up to host_threads threads
// (0: one per hardware thread), then one device pass for all of them.
P3G_API int p3g_verify_batch(p3g_ctx *x, const p3g_verify_job_c *jobs, uint64_t n, uint32_t host_threads,
                             int32_t *verdicts, p3g_verify_stats_c *stats) {
    if (!x || (n && (!jobs || !verdicts))) return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n; i++) {
        const p3g_verify_job_c &J = jobs[i];
        if (int e = p3g::verify_args_ok(&J.pcs, J.instances, J.n_instances, J.fields, J.n_fields, J.commits,
                                        J.n_commits, J.digest12, false))
            return e;
    }
    const unsigned th = host_threads ? host_threads : std::max(1u, std::thread::hardware_concurrency());
    {  // the canonical-word scan, one proof per task on the host threads
        std::atomic<uint64_t> next{0};
        std::atomic<bool> ok{true};
        auto scan = [&]() {
            for (uint64_t i; (i = next.fetch_add(1)) < n;) {
                const p3g_verify_job_c &J = jobs[i];
                if (!(p3g::words_canonical(J.fields, J.n_fields) && p3g::words_canonical(J.commits, 4 * J.n_commits) &&
                      p3g::words_canonical(J.digest12, 12)))
                    ok = false;
            }
        };
        std::vector<std::thread> ts;
        for (unsigned t = 1; t < std::min<uint64_t>(th, n); t++) ts.emplace_back(scan);
        scan();
        for (auto &t : ts) t.join();
        if (!ok) return p3g::ERR_INVALID;
    }
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        std::vector<std::vector<p3g::Instance>> ins(n);
        std::vector<p3g::vfy::ProofRef> ps(n);
        for (uint64_t i = 0; i < n; i++) {
            const p3g_verify_job_c &J = jobs[i];
            ins[i] = p3g::shapes_of(J.instances, J.n_instances);
            ps[i] = p3g::vfy::ProofRef{p3g::pcs_of(&J.pcs), ins[i].data(), ins[i].size(), J.fields, J.n_fields,
                                       J.commits, J.n_commits, J.digest12};
        }
        std::vector<int> v(n);
        p3g::vfy::Timing tm;
        if (n) p3g::vfy::verify_batch(x->c, ps, th, v.data(), &tm);
        for (uint64_t i = 0; i < n; i++) verdicts[i] = v[i];
        if (stats) *stats = p3g_verify_stats_c{tm.host_ms, tm.device_ms, tm.launches};
    })
}

// Lmcs::open_batch (p3-miden-lmcs/src/lmcs.rs:167-290) for a tree of height
// 2^log_height over matrices of the given widths, opened at strictly
// ascending indices: fields are the hinted rows (each matrix's row padded to
// the alignment, then salt_width salt words for a hiding tree), commits the
// streamed sibling digests. *verdict: P3G_ACCEPT, P3G_VERR_OPENING,
// P3G_VERR_ROOT or P3G_VERR_TRANSCRIPT.
P3G_API int p3g_lmcs_open_batch(p3g_ctx *x, const uint64_t *commit4, const uint64_t *widths, uint64_t n_mats,
                                uint32_t alignment, uint64_t salt_width, uint32_t log_height, const uint64_t *indices,
                                uint64_t n_idx, const uint64_t *fields, uint64_t n_fields, const uint64_t *commits,
                                uint64_t n_commits, int32_t *verdict) {
    if (!x || !commit4 || !verdict || (n_mats && !widths) || (n_idx && !indices) || (!fields && n_fields) ||
        (!commits && n_commits) || log_height > 40 || n_mats > 64 || salt_width > 4096)
        return p3g::ERR_INVALID;
    for (uint64_t i = 1; i < n_idx; i++)
        if (indices[i] <= indices[i - 1]) return p3g::ERR_INVALID;
    const uint64_t a = alignment ? alignment : 1;
    std::vector<uint32_t> w;
    for (uint64_t m = 0; m < n_mats; m++) {
        if (widths[m] > (1u << 24)) return p3g::ERR_INVALID;
        w.push_back((uint32_t)((widths[m] + a - 1) / a * a));
    }
    if (salt_width) w.push_back((uint32_t)salt_width);
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        *verdict = p3g::vfy::lmcs_open_batch(x->c, commit4, w, log_height,
                                             std::vector<uint64_t>(indices, indices + n_idx), fields, n_fields,
                                             commits, n_commits);
    })
}
