// C-ABI entry points for the whole proof and for the caller-side helpers
// (trace generation). Declarations and reference citations: include/p3g.h.
#pragma once
#include <cstdlib>

#include "capi_stage.cuh"
#include "trace_gen.cuh"
#include "prover.cuh"
#include "traces.cuh"

struct p3g_pcs_params_c {
    uint32_t log_blowup, log_folding_arity, log_final_degree;
    uint32_t folding_pow_bits, deep_pow_bits, num_queries, query_pow_bits;
};
struct p3g_sym_air {
    sym::Air a;
};
struct p3g_instance_c {
    int32_t air;
    int32_t trace_on_device;
    uint64_t height, width;
    const uint64_t *trace;
    const uint64_t *consts;
    uint64_t n_consts;
    const p3g_sym_air *sym;
    const uint64_t *public_values;
    uint64_t n_public_values;
    p3g::AuxFn aux_build;
    void *aux_user;
};
struct p3g_proof_c {
    uint64_t *fields;
    uint64_t n_fields;
    uint64_t *commits;
    uint64_t n_commits;
    uint64_t digest[12];
    double stage_ms[12];
    uint64_t gpu_launches;
    uint64_t h2d_bytes, d2h_bytes;
};

namespace p3g {
// Upload the Keccak round constants and rho offsets used by the constraint kernel.
inline void upload_keccak_tables();
inline void ensure_keccak_tables(int device) {
    static std::mutex mu;
    static bool done[64] = {false};
    std::lock_guard<std::mutex> lk(mu);
    if (device >= 0 && device < 64 && !done[device]) {
        upload_keccak_tables();
        done[device] = true;
    }
}
inline void upload_keccak_tables() {
    const keccak::Tables &T = keccak::tables();
    int rot[25];
    for (int x = 0; x < 5; x++)
        for (int y = 0; y < 5; y++) rot[x * 5 + y] = T.rot[x][y];
    CK(cudaMemcpyToSymbol(quot::c_keccak_rc, T.rc, sizeof(T.rc)));
    CK(cudaMemcpyToSymbol(quot::c_keccak_rot, rot, sizeof(rot)));
    CK(cudaMemcpyToSymbol(tgen::c_rc, T.rc, sizeof(T.rc)));
    CK(cudaMemcpyToSymbol(tgen::c_rot, rot, sizeof(rot)));
}

inline Instance to_instance(const p3g_instance_c &I) {
    Instance r{I.air, I.trace_on_device, I.height, I.width, I.trace, I.consts, I.n_consts};
    r.sym = I.sym ? &I.sym->a : nullptr;
    r.pub = I.public_values;
    r.n_pub = I.n_public_values;
    r.aux_build = I.aux_build;
    r.aux_user = I.aux_user;
    return r;
}
// The AIR-specific shape checks (width, constants, public values): the
// WidthMismatch / public-values checks of AirWitness and AirInstance
// (p3-miden-lifted-air/src/instance.rs:93-115).
inline int validate_air(const p3g_instance_c &I) {
    if (I.air == AIR_KECCAK) {
        if (I.width != (uint64_t)keccak::NCOLS) return ERR_VALIDATION;
    } else if (I.air == AIR_CUBIC) {
        if (I.width == 0 || !I.consts || I.n_consts != I.width) return ERR_VALIDATION;
    } else if (I.air == AIR_SYMBOLIC) {
        if (!I.sym) return ERR_INVALID;
        const sym::Desc &d = I.sym->a.d;
        if (I.width != d.main_width) return ERR_VALIDATION;
        if (I.n_public_values != d.num_public_values || (d.num_public_values && !I.public_values))
            return ERR_VALIDATION;
    } else {
        return ERR_VALIDATION;
    }
    return OK;
}
// Validation mirroring prove_multi's checks (prover/mod.rs:238-264,
// p3-miden-lifted-air/src/instance.rs:93-115) and PcsParams::new
// (p3-miden-lifted-fri/src/params.rs:170-204).
inline int validate(const p3g_pcs_params_c *pcs, const p3g_instance_c *inst, uint64_t n) {
    if (!pcs || !inst || n == 0 || n > 8) return ERR_INVALID;
    if (pcs->log_folding_arity < 1 || pcs->log_folding_arity > 3) return ERR_INVALID;
    if (pcs->log_blowup == 0 || pcs->log_blowup > 8) return ERR_INVALID;
    if (pcs->num_queries == 0) return ERR_INVALID;
    if (pcs->folding_pow_bits > 30 || pcs->deep_pow_bits > 30 || pcs->query_pow_bits > 30) return ERR_INVALID;
    uint64_t prev = 0;
    for (uint64_t i = 0; i < n; i++) {
        const p3g_instance_c &I = inst[i];
        if (!I.trace) return ERR_INVALID;
        if (I.height == 0 || (I.height & (I.height - 1))) return ERR_VALIDATION;
        if (I.height < prev) return ERR_VALIDATION;  // not ascending
        prev = I.height;
        if (int v = validate_air(I)) return v;
    }
    if (prev < 2) return ERR_VALIDATION;  // max trace height must be >= 2
    uint32_t log_qd = 0;
    for (uint64_t i = 0; i < n; i++) log_qd = std::max(log_qd, inst_log_qd(to_instance(inst[i])));
    if (log_qd > pcs->log_blowup) return ERR_VALIDATION;  // ConstraintDegreeTooHigh
    if (log_qd > 3) return ERR_VALIDATION;  // this library's bound: at most 8 quotient chunks (degree <= 9)
    if (log2u(prev) + pcs->log_blowup > 32) return ERR_INVALID;  // two-adicity of Goldilocks
    return OK;
}
}  // namespace p3g

P3G_API int p3g_prove(p3g_ctx *x, const p3g_pcs_params_c *pcs, const p3g_instance_c *inst, uint64_t n,
                      p3g_proof_c *out) {
    if (!x || !out) return p3g::ERR_INVALID;
    memset(out, 0, sizeof(*out));
    int v = p3g::validate(pcs, inst, n);
    if (v != p3g::OK) {
        x->c.last_error = "instance or parameter validation failed";
        return v;
    }
    try {
        CK(cudaSetDevice(x->c.device));
        p3g::bind_p2(x->c);
        p3g::ensure_keccak_tables(x->c.device);
        std::vector<p3g::Instance> ins(n);
        for (uint64_t i = 0; i < n; i++) ins[i] = p3g::to_instance(inst[i]);
        p3g::PcsParams pp{pcs->log_blowup,     pcs->log_folding_arity, pcs->log_final_degree, pcs->folding_pow_bits,
                          pcs->deep_pow_bits,  pcs->num_queries,       pcs->query_pow_bits};
        p3g::ProofOut po;
        p3g::prove(x->c, pp, ins.data(), n, po);
        out->n_fields = po.fields.size();
        out->n_commits = po.commits.size() / 4;
        out->fields = (uint64_t *)malloc(std::max<size_t>(1, po.fields.size()) * 8);
        out->commits = (uint64_t *)malloc(std::max<size_t>(1, po.commits.size()) * 8);
        if (!out->fields || !out->commits) throw std::bad_alloc();
        memcpy(out->fields, po.fields.data(), po.fields.size() * 8);
        memcpy(out->commits, po.commits.data(), po.commits.size() * 8);
        memcpy(out->digest, po.digest, sizeof(po.digest));
        for (int s = 0; s < 12; s++) out->stage_ms[s] = po.stage_ms[s];
        out->gpu_launches = po.launches;
        out->h2d_bytes = po.h2d;
        out->d2h_bytes = po.d2h;
    } catch (const p3g::CudaError &e) {
        x->c.last_error = e.what;
        return e.status;
    } catch (const std::bad_alloc &) {
        x->c.last_error = "host allocation failed";
        return p3g::ERR_OOM;
    }
    return p3g::OK;
}

// Wire format of a proof (StarkOutput: digest + TranscriptData,
// p3-miden-lifted-stark/src/proof.rs:39-44, p3-miden-transcript/src/data.rs:11-14),
// little-endian: "P3GPROOF", u32 version 1, u32 0, u64 n_fields, u64 n_commits,
// 12 digest words (a 128-byte header), then the field words, then the
// commitment words. The payload is TranscriptData's size_in_bytes
// (data.rs:46-48): 8 bytes per field element, 32 per commitment.
namespace p3g {
constexpr uint64_t kWireHeader = 128;
constexpr char kWireMagic[8] = {'P', '3', 'G', 'P', 'R', 'O', 'O', 'F'};
}  // namespace p3g
P3G_API uint64_t p3g_proof_wire_size(const p3g_proof_c *p) {
    return p ? p3g::kWireHeader + 8 * p->n_fields + 32 * p->n_commits : 0;
}
P3G_API int p3g_proof_serialize(const p3g_proof_c *p, uint8_t *buf, uint64_t cap, uint64_t *len) {
    if (!p || !len || (p->n_fields && !p->fields) || (p->n_commits && !p->commits)) return p3g::ERR_INVALID;
    const uint64_t n = p3g_proof_wire_size(p);
    *len = n;
    if (!buf || cap < n) return p3g::ERR_INVALID;
    const uint32_t ver[2] = {1, 0};
    const uint64_t counts[2] = {p->n_fields, p->n_commits};
    memcpy(buf, p3g::kWireMagic, 8);
    memcpy(buf + 8, ver, 8);
    memcpy(buf + 16, counts, 16);
    memcpy(buf + 32, p->digest, 96);
    if (p->n_fields) memcpy(buf + p3g::kWireHeader, p->fields, 8 * p->n_fields);
    if (p->n_commits) memcpy(buf + p3g::kWireHeader + 8 * p->n_fields, p->commits, 32 * p->n_commits);
    return p3g::OK;
}
// Parses a serialized proof into malloc'ed buffers (release with
// p3g_proof_free). P3G_ERR_INVALID for a wrong magic or version, a length
// that does not match the counts, or a word that is not a canonical field
// element.
P3G_API int p3g_proof_deserialize(const uint8_t *buf, uint64_t len, p3g_proof_c *out) {
    if (!buf || !out || len < p3g::kWireHeader) return p3g::ERR_INVALID;
    memset(out, 0, sizeof(*out));
    uint32_t ver[2];
    uint64_t counts[2];
    memcpy(ver, buf + 8, 8);
    memcpy(counts, buf + 16, 16);
    if (memcmp(buf, p3g::kWireMagic, 8) != 0 || ver[0] != 1 || ver[1] != 0) return p3g::ERR_INVALID;
    if (counts[0] > (len / 8) || counts[1] > (len / 32)) return p3g::ERR_INVALID;
    if (p3g::kWireHeader + 8 * counts[0] + 32 * counts[1] != len) return p3g::ERR_INVALID;
    const uint8_t *body = buf + p3g::kWireHeader;
    for (uint64_t i = 0; i < 12 + counts[0] + 4 * counts[1]; i++) {
        uint64_t w;
        memcpy(&w, i < 12 ? buf + 32 + 8 * i : body + 8 * (i - 12), 8);
        if (w >= gl::P) return p3g::ERR_INVALID;
    }
    out->fields = (uint64_t *)malloc(std::max<uint64_t>(1, counts[0]) * 8);
    out->commits = (uint64_t *)malloc(std::max<uint64_t>(1, counts[1]) * 32);
    if (!out->fields || !out->commits) {
        free(out->fields), free(out->commits);
        out->fields = out->commits = nullptr;
        return p3g::ERR_OOM;
    }
    out->n_fields = counts[0], out->n_commits = counts[1];
    memcpy(out->digest, buf + 32, 96);
    if (counts[0]) memcpy(out->fields, body, 8 * counts[0]);
    if (counts[1]) memcpy(out->commits, body + 8 * counts[0], 32 * counts[1]);
    return p3g::OK;
}

P3G_API void p3g_proof_free(p3g_proof_c *p) {
    if (!p) return;
    free(p->fields);
    free(p->commits);
    p->fields = p->commits = nullptr;
    p->n_fields = p->n_commits = 0;
}

P3G_API int p3g_keccak_inputs(uint64_t seed, uint64_t n_perms, uint64_t *out25) {
    if (!out25 && n_perms) return p3g::ERR_INVALID;
    p3g::keccak_inputs(seed, n_perms, out25);
    return p3g::OK;
}
P3G_API int p3g_keccak_trace(const uint64_t *inputs25, uint64_t n_perms, uint32_t log_height, uint64_t *out) {
    if (!out || (!inputs25 && n_perms) || log_height > 30) return p3g::ERR_INVALID;
    if (n_perms * 24 > (1ull << log_height)) return p3g::ERR_INVALID;
    p3g::keccak_trace(inputs25, n_perms, log_height, out);
    return p3g::OK;
}
// The same trace generated on the device from device-resident inputs, on the
// context's stream; returns once the trace is written.
P3G_API int p3g_keccak_trace_device(p3g_ctx *x, const uint64_t *d_inputs25, uint64_t n_perms, uint32_t log_height,
                                    uint64_t *d_out) {
    if (!x || !d_out || (!d_inputs25 && n_perms) || log_height > 30) return p3g::ERR_INVALID;
    if (n_perms * 24 > (1ull << log_height)) return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        p3g::ensure_keccak_tables(x->c.device);
        const uint64_t h = 1ull << log_height;
        tgen::keccak_trace_kernel<<<(unsigned)((h + 23) / 24), 128, 0, x->c.stream>>>(d_inputs25, n_perms, h, d_out);
        CK(cudaGetLastError());
        x->c.launches++;
        x->c.sync();
    })
}
P3G_API int p3g_cubic_trace(uint32_t log_height, uint64_t width, uint64_t seed, uint64_t *consts_out,
                            uint64_t *trace_out) {
    if (!consts_out || !trace_out || width == 0 || log_height > 30) return p3g::ERR_INVALID;
    p3g::cubic_trace(log_height, width, seed, consts_out, trace_out);
    return p3g::OK;
}
// The cubic AIR's trace generated on the device: k and row 0 drawn from
// SmallRng(seed) on the host (as p3g_cubic_trace), the forward iteration on
// the device into d_out (2^log_height x width, row-major); consts_out (host)
// receives k. Bit-identical to p3g_cubic_trace.
P3G_API int p3g_cubic_trace_device(p3g_ctx *x, uint32_t log_height, uint64_t width, uint64_t seed,
                                   uint64_t *consts_out, uint64_t *d_out) {
    if (!x || !consts_out || !d_out || width == 0 || width > tgen::kCubicMaxWidth || log_height > 30)
        return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        std::vector<uint64_t> kr(2 * width);
        p3g::cubic_trace(0, width, seed, kr.data(), kr.data() + width);  // k, then row 0
        memcpy(consts_out, kr.data(), width * 8);
        p3g::DBuf d = x->c.upload(kr);
        const int threads = (int)std::min<uint64_t>(1024, (width + 31) / 32 * 32);
        const size_t smem = 2 * width * 8;
        static std::atomic<uint64_t> attr_done{0};
        p3g::smem_attr_once(attr_done, tgen::cubic_trace_kernel, (int)(2 * tgen::kCubicMaxWidth * 8));
        tgen::cubic_trace_kernel<<<1, threads, smem, x->c.stream>>>(d.p + width, d.p, width, 1ull << log_height, d_out);
        CK(cudaGetLastError());
        x->c.launches++;
        x->c.sync();
    })
}
P3G_API uint64_t p3g_air_num_constraints(int32_t air, uint64_t width) { return p3g::air_num_constraints(air, width); }

// Proof-of-work witness search for a challenger state (GrindingChallenger::grind).
P3G_API int p3g_grind(p3g_ctx *x, const uint64_t *state12, const uint64_t *pending, uint32_t n_pending, uint32_t bits,
                      uint64_t *witness) {
    if (!x || !state12 || !witness || n_pending > 7 || (n_pending && !pending) || bits > 30) return p3g::ERR_INVALID;
    P3G_TRY(x, {
        if (bits == 0) {
            *witness = 0;
        } else {
            ::fri::GrindArgs g{};
            memcpy(g.state, state12, 96);
            for (uint32_t i = 0; i < n_pending; i++) g.pending[i] = pending[i];
            g.n_pending = n_pending;
            g.bits = bits;
            p3g::DBuf fb = x->c.alloc(1);
            uint64_t found = ~0ull;
            for (uint64_t base = 0; base < (1ull << 36) && found == ~0ull; base += (1ull << 22)) {
                CK(cudaMemsetAsync(fb.p, 0xff, 8, x->c.stream));
                g.base = base;
                g.count = 1ull << 22;
                g.found = (unsigned long long *)fb.p;
                ::fri::grind_kernel<<<148 * 8, 128, 0, x->c.stream>>>(g);
                CK(cudaGetLastError());
                x->c.d2h(x->c.stage(1), fb.p, 1);
                x->c.sync();
                found = x->c.pinned[0];
            }
            if (found == ~0ull) throw p3g::CudaError{p3g::ERR_TIMEOUT, "grind: search bound reached"};
            *witness = found;
        }
    })
}

// LmcsTree::prove_batch hints for sorted unique indices.
P3G_API int p3g_lmcs_prove_batch(p3g_ctx *x, const p3g_tree *t, const uint64_t *indices, uint64_t n,
                                 uint64_t *fields_out, uint64_t *n_fields, uint64_t *commits_out, uint64_t *n_commits) {
    if (!x || !t || !fields_out || !n_fields || !commits_out || !n_commits || (n && !indices)) return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n; i++) {
        if (indices[i] >= t->t.H) return p3g::ERR_INVALID;
        if (i && indices[i] <= indices[i - 1]) return p3g::ERR_INVALID;
    }
    P3G_TRY(x, {
        std::vector<uint64_t> idx(indices, indices + n);
        p3g::OpeningPlan p;
        p3g::plan_openings(t->t, idx, p);
        uint64_t nf = 0;
        for (auto &r : p.rows) nf += r.padded;
        if (nf > *n_fields || p.sibs.size() > *n_commits) throw p3g::CudaError{p3g::ERR_INVALID, "output buffers too small"};
        uint64_t of = 0, oc = 0;
        for (auto &r : p.rows) {
            CK(cudaMemcpyAsync(fields_out + of, r.src, r.len * 8, cudaMemcpyDeviceToHost, x->c.stream));
            x->c.sync();
            for (uint64_t k = r.len; k < r.padded; k++) fields_out[of + k] = 0;
            of += r.padded;
        }
        for (auto *s : p.sibs) {
            CK(cudaMemcpyAsync(commits_out + 4 * oc, s, 32, cudaMemcpyDeviceToHost, x->c.stream));
            oc++;
        }
        x->c.sync();
        *n_fields = of;
        *n_commits = oc;
    })
}

// LmcsTree::rows (p3-miden-lmcs/src/lifted_tree.rs:127-138): the row of each
// committed matrix at leaf `index` (lifted: row index >> log2(H / h)), each
// padded with zeros to the tree's alignment, concatenated into out; *n_words
// is the capacity on entry and the count on return.
P3G_API int p3g_lmcs_rows(p3g_ctx *x, const p3g_tree *t, uint64_t index, uint64_t *out, uint64_t *n_words) {
    if (!x || !t || !out || !n_words || index >= t->t.H) return p3g::ERR_INVALID;
    uint64_t need = 0;
    for (const p3g::Mat &m : t->t.mats) need += (m.w + t->t.alignment - 1) / t->t.alignment * t->t.alignment;
    if (need > *n_words) {
        *n_words = need;
        return p3g::ERR_INVALID;
    }
    P3G_TRY(x, {
        uint64_t off = 0;
        for (const p3g::Mat &m : t->t.mats) {
            const uint64_t r = index >> (t->t.depth - p3g::log2u(m.h));
            const uint64_t pad = (m.w + t->t.alignment - 1) / t->t.alignment * t->t.alignment;
            CK(cudaMemcpyAsync(out + off, m.d + r * m.w, m.w * 8, cudaMemcpyDeviceToHost, x->c.stream));
            for (uint64_t k = m.w; k < pad; k++) out[off + k] = 0;
            off += pad;
        }
        x->c.sync();
        *n_words = off;
    })
}

// FriFold::fold_matrix (p3-miden-lifted-fri/src/fri/fold/mod.rs:119-181,
// arity{2,4,8}.rs): d_in holds n = 2^log_n EF values of a FRI layer in
// bit-reversed order; row k (its 2^log_arity consecutive values) is the coset
// s*<w_a> with s = w_n^{bitrev(k)}, and folds with beta to
// (1/a) sum_j (beta/s)^j sum_t y_t w_a^{-jt} in d_out[k] (n / a EF). The
// layer's commitment is p3g_lmcs_build of d_in viewed as (n/a) x 2a with
// alignment 1 (fri/prover.rs:143-150).
P3G_API int p3g_fri_fold(p3g_ctx *x, const uint64_t *d_in, uint32_t log_n, uint32_t log_arity, const uint64_t *beta2,
                         uint64_t *d_out) {
    if (!x || !d_in || !d_out || !beta2 || log_arity < 1 || log_arity > 3 || log_n < log_arity || log_n > 32 ||
        beta2[0] >= gl::P || beta2[1] >= gl::P)
        return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        const p3g::TwTables &tw = x->c.twiddles(log_n);
        fri::FoldArgs fa{};
        fa.in = d_in;
        fa.n_out = 1ull << (log_n - log_arity);
        fa.log_a = log_arity;
        fa.log_nin = log_n;
        fa.log_n0 = log_n;
        fa.w0inv = ntt::PowTab{tw.inv_lo.p, tw.inv_hi.p, tw.lo_bits};
        fa.beta = gl::ef{beta2[0], beta2[1]};
        fa.beta_dev = nullptr;
        const uint64_t wi = gl::inv(gl::root(log_arity));
        uint64_t w = 1;
        for (int i = 0; i < 8; i++) fa.winv_a[i] = w, w = gl::mul(w, wi);
        fa.inv_a = gl::inv(1ull << log_arity);
        fa.out = d_out;
        fa.digests = nullptr;
        const uint64_t threads = (fa.n_out + (1ull << log_arity) - 1) >> log_arity;
        fri::fold_hash_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, x->c.stream>>>(fa);
        CK(cudaGetLastError());
        x->c.launches++;
        x->c.sync();
    })
}

// DEEP, the openings at the two out-of-domain points z_0, z_1
// (PointQuotients::new, p3-miden-lifted-fri/src/deep/interpolate.rs:81-109,
// and batch_eval_lifted, :123-201) over committed matrices: bit-reversed LDEs
// on g*K (heights h_m = the LDE heights, ascending; the largest is the LDE
// domain), log_blowup B. evals_out (host) receives 4 words per column, matrix
// by matrix: f(z_0) (c0, c1), f(z_1) (c0, c1).
P3G_API int p3g_deep_evals(p3g_ctx *x, const uint64_t *const *d_mats, const uint64_t *heights, const uint64_t *widths,
                           uint64_t n_mats, uint32_t log_blowup, const uint64_t *z4, uint64_t *evals_out) {
    if (!x || !d_mats || !heights || !widths || !z4 || !evals_out || n_mats == 0 || n_mats > 64 || log_blowup > 8)
        return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n_mats; i++)
        if (heights[i] == 0 || (heights[i] & (heights[i] - 1)) || (i && heights[i] < heights[i - 1]) ||
            (heights[i] >> log_blowup) == 0 || !d_mats[i] || widths[i] == 0)
            return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        std::vector<p3g::Mat> mats;
        std::vector<const p3g::Mat *> all;
        for (uint64_t i = 0; i < n_mats; i++) mats.push_back({d_mats[i], heights[i], widths[i]});
        for (auto &m : mats) all.push_back(&m);
        const gl::ef zs[2] = {gl::ef{z4[0], z4[1]}, gl::ef{z4[2], z4[3]}};
        p3g::Launcher L{x->c};
        p3g::DeepOpen st;
        std::vector<uint64_t> ev = p3g::deep_evals(x->c, L, all, log_blowup, p3g::log2u(heights[n_mats - 1]), zs, 1,
                                                   st, nullptr);
        memcpy(evals_out, ev.data(), ev.size() * 8);
        x->c.launches += L.n;
    })
}

// DEEP, the quotient polynomial (DeepPoly::from_evals + accumulate_matrices,
// p3-miden-lifted-fri/src/deep/prover.rs:106-364): with evals from
// p3g_deep_evals, the column challenge alpha2 and the point challenge beta2,
// the reduced openings f_red(z_j) and coefficients -alpha^{W-1-c} run over
// the columns padded to `alignment` (the LMCS alignment; padding columns are
// zero), and d_out receives Q(x) = sum_j beta^j (f_red(z_j) - f_red(x)) /
// (z_j - x) on the LDE domain, bit-reversed (n EF, n = the largest height).
P3G_API int p3g_deep_quotient(p3g_ctx *x, const uint64_t *const *d_mats, const uint64_t *heights,
                              const uint64_t *widths, uint64_t n_mats, uint32_t log_blowup, uint32_t alignment,
                              const uint64_t *z4, const uint64_t *evals, const uint64_t *alpha2,
                              const uint64_t *beta2, uint64_t *d_out) {
    if (!x || !d_mats || !heights || !widths || !z4 || !evals || !alpha2 || !beta2 || !d_out || n_mats == 0 ||
        n_mats > 16 || log_blowup > 8 || alignment == 0 || alignment > 64)
        return p3g::ERR_INVALID;
    for (uint64_t i = 0; i < n_mats; i++)
        if (heights[i] == 0 || (heights[i] & (heights[i] - 1)) || (i && heights[i] < heights[i - 1]) ||
            (heights[i] >> log_blowup) == 0 || !d_mats[i] || widths[i] == 0)
            return p3g::ERR_INVALID;
    P3G_TRY(x, {
        CK(cudaSetDevice(x->c.device));
        std::vector<p3g::Mat> mats;
        std::vector<const p3g::Mat *> all;
        uint64_t total_w = 0;
        for (uint64_t i = 0; i < n_mats; i++) mats.push_back({d_mats[i], heights[i], widths[i]}), total_w += widths[i];
        for (auto &m : mats) all.push_back(&m);
        const gl::ef zs[2] = {gl::ef{z4[0], z4[1]}, gl::ef{z4[2], z4[3]}};
        const uint32_t log_lde = p3g::log2u(heights[n_mats - 1]);
        p3g::Launcher L{x->c};
        p3g::DeepOpen st;
        // the point quotients and weights of the opening, then the assembly
        (void)p3g::deep_evals(x->c, L, all, log_blowup, log_lde, zs, alignment, st, nullptr);
        std::vector<uint64_t> ev(evals, evals + 4 * total_w);
        p3g::DBuf layer = p3g::deep_assemble(x->c, L, all, log_lde, ev, gl::ef{alpha2[0], alpha2[1]},
                                             gl::ef{beta2[0], beta2[1]}, st);
        CK(cudaMemcpyAsync(d_out, layer.p, (2ull << log_lde) * 8, cudaMemcpyDeviceToDevice, x->c.stream));
        x->c.sync();
        x->c.launches += L.n;
    })
}

// ------------------------------------------------------------ symbolic AIRs
struct p3g_sym_node_c {
    uint32_t op, a, b, pad;
    uint64_t value;
};
struct p3g_air_desc_c {
    uint32_t main_width, aux_width, num_randomness, num_aux_values, num_public_values, num_periodic;
    const uint64_t *periodic_lengths;
    const uint64_t *periodic_values;
    const p3g_sym_node_c *nodes;
    uint64_t n_nodes;
    const uint32_t *constraints;
    const uint8_t *is_ext;
    uint64_t n_constraints;
};
namespace p3g {
inline int desc_from_c(const p3g_air_desc_c *c, sym::Desc &d, std::string &why) {
    if (!c || (c->n_nodes && !c->nodes) || (c->n_constraints && (!c->constraints || !c->is_ext)) ||
        (c->num_periodic && (!c->periodic_lengths || !c->periodic_values)) || c->n_nodes > (1ull << 24) ||
        c->n_constraints > (1ull << 24) || c->num_periodic > 4096)
        return ERR_INVALID;
    d.main_width = c->main_width, d.aux_width = c->aux_width, d.num_randomness = c->num_randomness;
    d.num_aux_values = c->num_aux_values, d.num_public_values = c->num_public_values, d.num_periodic = c->num_periodic;
    d.periodic_lengths.assign(c->periodic_lengths, c->periodic_lengths + c->num_periodic);
    uint64_t total = 0;
    for (uint64_t p : d.periodic_lengths) {
        if (p > (1ull << 30)) return ERR_INVALID;
        total += p;
    }
    d.periodic_values.assign(c->periodic_values, c->periodic_values + total);
    d.nodes.resize(c->n_nodes);
    if (c->n_nodes) memcpy(d.nodes.data(), c->nodes, c->n_nodes * sizeof(sym::Node));
    d.constraints.assign(c->constraints, c->constraints + c->n_constraints);
    d.is_ext.assign(c->is_ext, c->is_ext + c->n_constraints);
    if (const char *e = sym::validate(d)) {
        why = e;
        return ERR_VALIDATION;
    }
    return OK;
}
}  // namespace p3g

// The analysis alone (no device, no compilation): degree and layout.
P3G_API int p3g_air_analyse(const p3g_air_desc_c *desc, uint32_t *max_degree, uint32_t *log_quotient_degree,
                            uint64_t *n_base, uint64_t *n_ext) {
    sym::Air A;
    std::string why;
    if (int v = p3g::desc_from_c(desc, A.d, why)) return v;
    sym::analyse(A);
    if (max_degree) *max_degree = A.max_degree;
    if (log_quotient_degree) *log_quotient_degree = A.log_qd;
    if (n_base) *n_base = A.base_idx.size();
    if (n_ext) *n_ext = A.ext_idx.size();
    return p3g::OK;
}

// The generated kernel source of an AIR (no device needed); *len = its size
// plus the terminating zero, P3G_ERR_INVALID when cap is smaller.
P3G_API int p3g_air_generate_source(const p3g_air_desc_c *desc, char *buf, uint64_t cap, uint64_t *len) {
    if (!len) return p3g::ERR_INVALID;
    sym::Air A;
    std::string why;
    if (int v = p3g::desc_from_c(desc, A.d, why)) return v;
    sym::analyse(A);
    const std::string src = sym::generate(A);
    *len = src.size() + 1;
    if (!buf || cap < *len) return p3g::ERR_INVALID;
    memcpy(buf, src.c_str(), src.size() + 1);
    return p3g::OK;
}

// Generate and compile (NVRTC, sm_<cc>) without a device: 0 when the
// kernel compiles; *cubin_bytes receives its size.
P3G_API int p3g_air_compile_check(const p3g_air_desc_c *desc, int32_t cc, uint64_t *cubin_bytes) {
    sym::Air A;
    std::string why;
    if (int v = p3g::desc_from_c(desc, A.d, why)) return v;
    try {
        sym::analyse(A);
        sym::split_chunks(A);
        sym::compile_cubins(A, cc);
    } catch (const p3g::CudaError &e) {
        return e.status;
    }
    if (cubin_bytes) {
        *cubin_bytes = 0;
        for (auto &c : A.cubins) *cubin_bytes += c.size();
    }
    return p3g::OK;
}

P3G_API int p3g_air_create(p3g_ctx *x, const p3g_air_desc_c *desc, p3g_sym_air **out) {
    if (!x || !out) return p3g::ERR_INVALID;
    *out = nullptr;
    p3g_sym_air *a = new p3g_sym_air();
    std::string why;
    if (int v = p3g::desc_from_c(desc, a->a.d, why)) {
        x->c.last_error = "symbolic AIR rejected: " + why;
        delete a;
        return v;
    }
    try {
        CK(cudaSetDevice(x->c.device));
        sym::analyse(a->a);
        if (x->c.air_chunk_nodes) a->a.chunk_nodes = x->c.air_chunk_nodes;
        sym::split_chunks(a->a);
        sym::compile(a->a, x->c.device);
    } catch (const p3g::CudaError &e) {
        x->c.last_error = e.what;
        delete a;
        return e.status;
    }
    *out = a;
    return p3g::OK;
}
P3G_API uint32_t p3g_air_log_quotient_degree(const p3g_sym_air *a) { return a ? a->a.log_qd : 0; }
P3G_API uint32_t p3g_air_max_degree(const p3g_sym_air *a) { return a ? a->a.max_degree : 0; }
P3G_API uint64_t p3g_air_num_constraints_of(const p3g_sym_air *a) { return a ? a->a.d.constraints.size() : 0; }
P3G_API uint64_t p3g_air_num_kernels(const p3g_sym_air *a) { return a ? a->a.kernels.size() : 0; }
// ConstraintLayout: base_indices / ext_indices in emission order; *n_base and
// *n_ext are capacities on entry and counts on return.
P3G_API int p3g_air_layout(const p3g_sym_air *a, uint64_t *base_idx, uint64_t *n_base, uint64_t *ext_idx, uint64_t *n_ext) {
    if (!a || !n_base || !n_ext) return p3g::ERR_INVALID;
    const uint64_t nb = a->a.base_idx.size(), ne = a->a.ext_idx.size();
    if ((nb && (!base_idx || *n_base < nb)) || (ne && (!ext_idx || *n_ext < ne))) {
        *n_base = nb, *n_ext = ne;
        return p3g::ERR_INVALID;
    }
    if (nb) memcpy(base_idx, a->a.base_idx.data(), nb * 8);
    if (ne) memcpy(ext_idx, a->a.ext_idx.data(), ne * 8);
    *n_base = nb, *n_ext = ne;
    return p3g::OK;
}
P3G_API void p3g_air_free(p3g_sym_air *a) { delete a; }
