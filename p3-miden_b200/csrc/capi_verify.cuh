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

P3G_API int p3g_verify(p3g_ctx *x, const p3g_pcs_params_c *pcs, const p3g_instance_c *inst, uint64_t n,
                       const uint64_t *fields, uint64_t n_fields, const uint64_t *commits, uint64_t n_commits,
                       const uint64_t *digest12, int32_t *verdict, p3g_verify_stats_c *stats) {
    if (!x || !pcs || !inst || !digest12 || !verdict || n == 0 || n > 8) return p3g::ERR_INVALID;
    if ((!fields && n_fields) || (!commits && n_commits)) return p3g::ERR_INVALID;
    if (pcs->log_folding_arity < 1 || pcs->log_folding_arity > 3 || pcs->log_blowup == 0 || pcs->log_blowup > 8 ||
        pcs->num_queries == 0 || pcs->folding_pow_bits > 30 || pcs->deep_pow_bits > 30 || pcs->query_pow_bits > 30)
        return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n; i++) {
        const p3g_instance_c &I = inst[i];
        if (I.height > (1ull << 30)) return p3g::ERR_INVALID;
        if (I.air == p3g::AIR_KECCAK) {
            if (I.width != (uint64_t)p3g::keccak::NCOLS) return p3g::ERR_VALIDATION;
        } else if (I.air == p3g::AIR_CUBIC) {
            if (I.width == 0 || !I.consts || I.n_consts != I.width) return p3g::ERR_VALIDATION;
        } else {
            return p3g::ERR_VALIDATION;
        }
    }
    // transcript words are field elements: canonical, below p
    for (uint64_t i = 0; i < n_fields; i++)
        if (fields[i] >= gl::P) return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < 4 * n_commits; i++)
        if (commits[i] >= gl::P) return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        p3g::ensure_keccak_tables(x->c.device);
        std::vector<p3g::Instance> ins(n);
        for (uint64_t i = 0; i < n; i++)
            ins[i] = {inst[i].air, 0, inst[i].height, inst[i].width, nullptr, inst[i].consts, inst[i].n_consts};
        p3g::PcsParams pp{pcs->log_blowup,    pcs->log_folding_arity, pcs->log_final_degree, pcs->folding_pow_bits,
                          pcs->deep_pow_bits, pcs->num_queries,       pcs->query_pow_bits};
        p3g::vfy::Timing tm;
        *verdict = p3g::vfy::verify(x->c, pp, ins.data(), n, fields, n_fields, commits, n_commits, digest12, &tm);
        if (stats) *stats = p3g_verify_stats_c{tm.host_ms, tm.device_ms, tm.launches};
    })
}
