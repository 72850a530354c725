// prove_multi on one device: the protocol control flow of
// p3-miden-lifted-stark/src/prover/mod.rs:223-461 with every O(n) stage on
// the GPU and the transcript on the host.
#pragma once
#include <algorithm>
#include <chrono>
#include <set>

#include "context.cuh"
#include "deep.cuh"
#include "fri.cuh"
#include "quotient.cuh"
#include "symair.cuh"
#include "transcript.cuh"

namespace p3g {

enum Air : int { AIR_CUBIC = 1, AIR_KECCAK = 2, AIR_SYMBOLIC = 3 };

// AuxBuilder::build_aux_trace (p3-miden-lifted-air/src/auxiliary/builder.rs:16-37):
// writes the instance's aux trace (height x aux_width EF, 2 words each,
// row-major, host memory the library provides) and its aux values
// (num_aux_values EF); 0 = success.
typedef int (*AuxFn)(void *user, uint64_t instance, const uint64_t *main_trace, const uint64_t *randomness,
                     uint64_t n_randomness, uint64_t height, uint64_t *aux_out, uint64_t *aux_values_out);

struct PcsParams {
    uint32_t log_blowup, log_folding_arity, log_final_degree;
    uint32_t folding_pow_bits, deep_pow_bits, num_queries, query_pow_bits;
};

struct Instance {
    int32_t air;
    int32_t trace_on_device;
    uint64_t height, width;
    const uint64_t *trace;
    const uint64_t *consts;
    uint64_t n_consts;
    const sym::Air *sym = nullptr;     // AIR_SYMBOLIC
    const uint64_t *pub = nullptr;     // AirWitness::public_values
    uint64_t n_pub = 0;
    AuxFn aux_build = nullptr;         // null: the all-zero aux trace
    void *aux_user = nullptr;
};

// LiftedAir properties. The built-in AIRs declare the examples' dummy aux
// trace: one EF column, one challenge, no aux values
// (p3-miden-lifted-examples/src/lib.rs:93-103).
inline uint64_t inst_aux_width(const Instance &I) { return I.air == AIR_SYMBOLIC ? I.sym->d.aux_width : 1; }
inline uint64_t inst_num_randomness(const Instance &I) { return I.air == AIR_SYMBOLIC ? I.sym->d.num_randomness : 1; }
inline uint64_t inst_num_aux_values(const Instance &I) { return I.air == AIR_SYMBOLIC ? I.sym->d.num_aux_values : 0; }

struct ProofOut {
    std::vector<uint64_t> fields, commits;
    uint64_t digest[12];
    double stage_ms[12] = {0};  // [8] = main-trace LDE kernel time (CUDA events on the LDE stream)
    uint64_t launches = 0, h2d = 0, d2h = 0;
};

inline uint64_t air_num_constraints(int air, uint64_t width) {
    if (air == AIR_CUBIC) return width;
    if (air == AIR_KECCAK) return 3182;
    return 0;
}
// Both built-in AIRs have maximal constraint degree 3 (is_transition counts
// 0, is_first_row 1): log2_ceil(3 - 1) = 1 (p3-miden-lifted-air/src/air.rs:225-247).
inline uint32_t air_log_quotient_degree(int air) {
    (void)air;
    return 1;
}
inline uint32_t inst_log_qd(const Instance &I) {
    return I.air == AIR_SYMBOLIC ? I.sym->log_qd : air_log_quotient_degree(I.air);
}
inline uint64_t inst_num_constraints(const Instance &I) {
    return I.air == AIR_SYMBOLIC ? I.sym->d.constraints.size() : air_num_constraints(I.air, I.width);
}

struct Launcher {
    Ctx &ctx;
    uint64_t n = 0;
    template <typename K, typename... Args>
    void operator()(K kernel, dim3 grid, dim3 block, size_t smem, Args... args) {
        kernel<<<grid, block, smem, ctx.stream>>>(args...);
        CK(cudaGetLastError());
        n++;
    }
};

inline unsigned blocks_for(uint64_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

// Query-phase openings of one tree (p3-miden-lmcs/src/lifted_tree.rs:157-224):
// rows per unique index per matrix (padded to the alignment), then sibling
// digests level by level, left to right.
struct OpeningPlan {
    struct RowRef {
        const uint64_t *src;
        uint64_t len, padded;
    };
    std::vector<RowRef> rows;
    std::vector<const uint64_t *> sibs;
};
inline void plan_openings(const Tree &t, const std::vector<uint64_t> &idx, OpeningPlan &p) {
    for (uint64_t i : idx) {
        for (const Mat &m : t.mats) {
            uint32_t lift = t.depth - log2u(m.h);
            uint64_t r = i >> lift;
            uint64_t pad = (m.w + t.alignment - 1) / t.alignment * t.alignment;
            p.rows.push_back({m.d + r * m.w, m.w, pad});
        }
        if (t.salt.d) p.rows.push_back({t.salt.d + i * t.salt.w, t.salt.w, t.salt.w});  // salt: unpadded
    }
    std::vector<uint64_t> known = idx;
    for (uint32_t l = 0; l < t.depth; l++) {
        std::vector<uint64_t> parents;
        for (size_t i = 0; i < known.size(); i++) {
            uint64_t pos = known[i], par = pos >> 1;
            if (!parents.empty() && parents.back() == par) continue;
            bool has_l, has_r;
            if ((pos & 1) == 0) {
                has_l = true;
                has_r = i + 1 < known.size() && known[i + 1] == pos + 1;
            } else {
                has_l = false;
                has_r = true;
            }
            const uint64_t *layer = t.layers.p + 4 * t.layer_off(l);
            if (has_l && !has_r) p.sibs.push_back(layer + 4 * (2 * par + 1));
            if (!has_l && has_r) p.sibs.push_back(layer + 4 * (2 * par));
            parents.push_back(par);
        }
        known.swap(parents);
    }
}

struct Seg {
    const uint64_t *src;
    uint64_t len;
    uint64_t dst;
};
__global__ void gather_kernel(const Seg *segs, uint64_t n, uint64_t *out) {
    for (uint64_t s = blockIdx.x; s < n; s += gridDim.x) {
        Seg g = segs[s];
        for (uint64_t i = threadIdx.x; i < g.len; i += blockDim.x) out[g.dst + i] = g.src[i];
    }
}

// Upload (or alias) a trace, returning a device pointer.
inline const uint64_t *trace_on_device(Ctx &ctx, const Instance &in, DBuf &hold, ProofOut &po) {
    if (in.trace_on_device) return in.trace;
    size_t words = in.height * in.width;
    hold = ctx.alloc(words);
    CK(cudaMemcpyAsync(hold.p, in.trace, words * 8, cudaMemcpyHostToDevice, ctx.stream));
    po.h2d += words * 8;
    return hold.p;
}

// Main-trace commitment, pipelined over column slabs (slab widths are
// multiples of 8, so absorbing a row slab by slab equals absorbing it whole):
//   copy stream : H2D of slab s of a host trace (pinned memory: 2D copy)
//   LDE stream  : coset LDE of slab s straight into its columns of the LDE
//   ctx stream  : leaf-sponge absorption of slab s into the running states
// The LDE (HBM-bound) of slab s+1 and the copy of slab s+2 run under the
// hash (integer-bound) of slab s. `ev_lde_done` is recorded on the context
// stream once every LDE slab is written (stage timing).
// cm[i], when not null, receives a column-major copy of the first
// h_i << log_qd_i LDE rows of trace i (written by the leaf kernels as they
// absorb the rows; the generated constraint kernels read it).
inline void commit_main_pipelined(Ctx &ctx, const Instance *inst, size_t n_inst, uint32_t lb, uint32_t log_max_h,
                                  std::vector<DBuf> &main_lde, std::vector<Mat> &main_mats, Tree &t, ProofOut &po,
                                  cudaEvent_t ev_lde_done, const std::vector<uint64_t *> &cm) {
    ctx.pipeline_streams();
    const uint64_t H = inst[n_inst - 1].height << lb;
    t.alignment = 8;
    t.H = H;
    t.depth = log2u(H);
    t.layers = ctx.alloc((2 * H - 1) * 4);
    struct Slab {
        size_t trace;
        uint64_t c0, w;
    };
    std::vector<Slab> slabs;
    uint64_t max_slab_hw = 0, max_state_h = 0;
    for (size_t i = 0; i < n_inst; i++) {
        uint64_t w = inst[i].width, h = inst[i].height;
        if (!inst[i].trace_on_device && w >= 256) {
            // a wide host trace: slabs that grow geometrically (x1.5, multiples of
            // the rate 8) from about 1/64 of the width, so that only the small
            // first slab's upload is exposed and each later upload (PCIe) fits
            // under the LDE and hash of the slab before it (about 1.6x the
            // upload time per column on a B200 at blowup 2, more at larger
            // blowups)
            uint64_t cur = std::max<uint64_t>(8, (w / 64 + 7) / 8 * 8);
            for (uint64_t c0 = 0; c0 < w;) {
                const uint64_t take = std::min(cur, w - c0);
                slabs.push_back({i, c0, take});
                max_slab_hw = std::max(max_slab_hw, h * take);
                c0 += take;
                cur = (cur * 3 / 2 + 7) / 8 * 8;
            }
        } else {
            uint64_t sw = w >= 256 ? ((w + 7) / 8 + 7) / 8 * 8 : w;  // about 8 slabs for wide traces
            // tuned width (a multiple of the rate, 8) for device-resident traces
            if (ctx.slab_cols) sw = std::min<uint64_t>(w, ctx.slab_cols);
            for (uint64_t c0 = 0; c0 < w; c0 += sw) {
                slabs.push_back({i, c0, std::min(sw, w - c0)});
                max_slab_hw = std::max(max_slab_hw, h * std::min(sw, w - c0));
            }
        }
        main_lde[i] = ctx.alloc((h << lb) * w);
        main_mats.push_back({main_lde[i].p, h << lb, w});
        max_state_h = std::max(max_state_h, h << lb);
    }
    const bool any_host = [&] {
        for (size_t i = 0; i < n_inst; i++)
            if (!inst[i].trace_on_device) return true;
        return false;
    }();
    DBuf tmp = ctx.alloc(max_slab_hw);
    DBuf inbuf[2];
    if (any_host) inbuf[0] = ctx.alloc(max_slab_hw), inbuf[1] = ctx.alloc(max_slab_hw);
    DBuf st[2];
    if (slabs.size() > 1) st[0] = ctx.alloc(max_state_h * 12), st[1] = ctx.alloc(max_state_h * 12);
    std::vector<LdePlan> plans;
    for (size_t i = 0; i < n_inst; i++)
        plans.push_back(lde_plan(ctx, inst[i].height, lb, gl::exp2k(gl::GEN, log_max_h - log2u(inst[i].height))));
    // allocations and tables are complete once the context stream drained (lde_plan syncs it)
    std::vector<cudaEvent_t> ev_copy(slabs.size()), ev_lde(slabs.size()), ev_t0(slabs.size());
    for (size_t s = 0; s < slabs.size(); s++) {
        CK(cudaEventCreateWithFlags(&ev_copy[s], cudaEventDisableTiming));
        CK(cudaEventCreate(&ev_lde[s]));
        CK(cudaEventCreate(&ev_t0[s]));
    }
    // 1) copies and LDEs of every slab (copy / LDE streams)
    for (size_t s = 0; s < slabs.size(); s++) {
        const Slab &sl = slabs[s];
        const Instance &I = inst[sl.trace];
        const uint64_t h = I.height, w = I.width;
        const uint64_t *src;
        uint64_t ld_in;
        if (I.trace_on_device) {
            src = I.trace + sl.c0;
            ld_in = w;
        } else {
            uint64_t *dst = inbuf[s & 1].p;
            if (s >= 2) CK(cudaStreamWaitEvent(ctx.copy_stream, ev_lde[s - 2], 0));  // buffer reuse
            CK(cudaMemcpy2DAsync(dst, sl.w * 8, I.trace + sl.c0, w * 8, sl.w * 8, h, cudaMemcpyHostToDevice,
                                 ctx.copy_stream));
            po.h2d += h * sl.w * 8;
            CK(cudaEventRecord(ev_copy[s], ctx.copy_stream));
            CK(cudaStreamWaitEvent(ctx.lde_stream, ev_copy[s], 0));
            src = dst;
            ld_in = sl.w;
        }
        CK(cudaEventRecord(ev_t0[s], ctx.lde_stream));
        lde_run(ctx, plans[sl.trace], src, ld_in, sl.w, main_lde[sl.trace].p + sl.c0, w, tmp.p, ctx.lde_stream);
        CK(cudaEventRecord(ev_lde[s], ctx.lde_stream));
    }
    // 2) leaf absorption per slab (context stream). With host traces each slab
    // starts as soon as its LDE is written, hiding the upload under the hash;
    // with device-resident traces both phases are integer-bound, so the hash
    // starts after the whole LDE and each phase runs alone.
    const uint64_t *prev = nullptr;
    uint32_t prev_log = 0;
    cudaEvent_t ev_leaf[2];
    CK(cudaEventCreate(&ev_leaf[0]));
    CK(cudaEventCreate(&ev_leaf[1]));
    for (size_t s = 0; s < slabs.size(); s++) {
        const Slab &sl = slabs[s];
        const Instance &I = inst[sl.trace];
        const uint64_t h = I.height, w = I.width;
        CK(cudaStreamWaitEvent(ctx.stream, any_host ? ev_lde[s] : ev_lde[slabs.size() - 1], 0));
        if (s == 0) CK(cudaEventRecord(ev_leaf[0], ctx.stream));
        merkle::ClassArgs a{};
        a.n_mats = 1;
        a.data[0] = main_lde[sl.trace].p + sl.c0;
        a.width[0] = sl.w;
        a.ld[0] = w;
        a.log_h = log2u(h << lb);
        a.prev = prev;
        a.prev_log_h = prev_log;
        if (cm[sl.trace]) {
            const uint64_t qh = h << inst_log_qd(I);
            a.cm = cm[sl.trace] + sl.c0 * qh;
            a.cm_ld = qh;
            a.cm_rows = qh;
        }
        const bool last = s + 1 == slabs.size();
        uint64_t *out_states = st[s & 1].p;
        a.states_out = last ? nullptr : out_states;
        a.digests_out = last ? t.layers.p : nullptr;
        launch_leaf_class(ctx, a, h << lb);
        prev = out_states;
        prev_log = a.log_h;
    }
    CK(cudaEventRecord(ev_leaf[1], ctx.stream));
    CK(cudaEventRecord(ev_lde_done, ctx.lde_stream));  // the last LDE slab is written
    finish_tree(ctx, t);
    t.mats = main_mats;
    double lde_ms = 0;
    for (size_t s = 0; s < slabs.size(); s++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev_t0[s], ev_lde[s]));
        lde_ms += ms;
        cudaEventDestroy(ev_copy[s]);
        cudaEventDestroy(ev_lde[s]);
        cudaEventDestroy(ev_t0[s]);
    }
    po.stage_ms[8] = lde_ms;
    // leaf sponge: the span of its launches on the context stream (with a
    // host trace the span also holds waits for slab LDEs) and their count
    float leaf_ms = 0;
    CK(cudaEventElapsedTime(&leaf_ms, ev_leaf[0], ev_leaf[1]));
    po.stage_ms[9] = leaf_ms;
    po.stage_ms[10] = (double)slabs.size();
    cudaEventDestroy(ev_leaf[0]);
    cudaEventDestroy(ev_leaf[1]);
}

// Constraint evaluation of a symbolic AIR on gJ with its generated kernel
// (symair.cuh): one thread per point, acc[m] += sum_k alpha^{K-1-k} C_k(x_m).
// The kernels read column-major copies of gJ's rows of the main and aux LDEs
// (cm: the main part from the main commit's leaf kernels, the aux part from one
// transpose), so that every cell load of a warp is one 256-byte run.
// Periodic columns: PeriodicLde::build on the quotient coset (blowup D,
// shift (g^{2^lift})^{h / max_period}, natural order; periodic.rs:49-98).
inline void eval_symbolic(Ctx &ctx, const Instance &I, uint64_t *cm, const uint64_t *aux_lde,
                          uint32_t log_h, uint32_t log_qd, uint32_t log_max_h, const std::vector<uint64_t> &rnd,
                          const std::vector<uint64_t> &auxv, const std::vector<uint64_t> &alpha_pows, uint64_t *acc) {
    const sym::Air &A = *I.sym;
    const sym::Desc &d = A.d;
    if (A.device != ctx.device) throw CudaError{ERR_INVALID, "symbolic AIR compiled for another device"};
    std::vector<uint64_t> k(A.kl.words, 0);
    for (uint64_t i = 0; i < d.num_public_values; i++) k[A.kl.pub + i] = I.pub[i] % gl::P;
    for (uint64_t i = 0; i < 2ull * d.num_randomness; i++) k[A.kl.rnd + i] = rnd[i];
    for (uint64_t i = 0; i < 2ull * d.num_aux_values; i++) k[A.kl.auxv + i] = auxv[i];
    for (size_t i = 0; i < alpha_pows.size(); i++) k[A.kl.alpha + i] = alpha_pows[i];
    DBuf dk = ctx.upload(k.empty() ? std::vector<uint64_t>{0} : k);
    const uint64_t h = 1ull << log_h, qh = h << log_qd, D = 1ull << log_qd;
    const uint64_t shift = gl::exp2k(gl::GEN, log_max_h - log_h);
    DBuf per_nat;
    uint64_t per_h = 0;
    if (d.num_periodic) {
        uint64_t max_p = 0;
        std::vector<uint64_t> rep = sym::periodic_matrix(d, max_p);
        const uint32_t log_p = log2u(max_p);
        per_h = max_p << log_qd;
        DBuf drep = ctx.upload(rep), brev = ctx.alloc(per_h * d.num_periodic), tmp = ctx.alloc(max_p * d.num_periodic);
        per_nat = ctx.alloc(per_h * d.num_periodic);
        coset_lde(ctx, drep.p, d.num_periodic, max_p, d.num_periodic, log_qd, gl::exp2k(shift, log_h - log_p), brev.p,
                  tmp.p);
        const uint64_t n = per_h * d.num_periodic;
        bitrev_rows_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx.stream>>>(brev.p, per_nat.p, log_p + log_qd,
                                                                                 d.num_periodic);
        CK(cudaGetLastError());
        ctx.launches++;
        ctx.sync();
    }
    const TwTables &twq = ctx.twiddles(log_h + log_qd);
    // the generated kernels read gJ's rows of the LDEs column-major: the main
    // part of cm was written by the main commit's leaf kernels; the aux part
    // is copied here
    const uint64_t aw2 = (d.aux_width && aux_lde) ? 2 * d.aux_width : 0;
    uint64_t *main_cm = cm, *aux_cm = aw2 ? cm + qh * I.width : nullptr;
    if (aw2) transpose(ctx, aux_lde, aw2, aux_cm, qh, aw2);
    sym::KArgs a{};
    a.main = main_cm;
    a.main_w = I.width;
    a.aux = aux_cm;
    a.aux_w2 = 2 * d.aux_width;
    a.per = per_nat.p;
    a.per_h = per_h ? per_h : 1;
    a.per_w = d.num_periodic;
    a.k = dk.p;
    a.qh = qh;
    a.log_qh = log_h + log_qd;
    a.D = D;
    a.shift = shift;
    a.wq_lo = twq.fwd_lo.p;
    a.wq_hi = twq.fwd_hi.p;
    a.wq_lo_bits = twq.lo_bits;
    a.omega_h_inv = gl::inv(gl::root(log_h));
    {
        uint64_t s_pow_n = gl::exp2k(shift, log_h), wd = gl::root(log_qd), x = 1;
        for (uint64_t t = 0; t < D && t < 8; t++) a.zh[t] = gl::sub(gl::mul(s_pow_n, x), 1), x = gl::mul(x, wd);
    }
    a.acc = acc;
    void *args[] = {&a};
    for (cudaKernel_t k : A.kernels) {  // one launch per constraint chunk, each adding its part of the fold
        CK(cudaLaunchKernel((const void *)k, dim3((unsigned)((qh + 127) / 128)), dim3(128), args, 0, ctx.stream));
        ctx.launches++;
    }
    ctx.sync();  // keep the constant block and the periodic table alive until the kernel ran
}

// DEEP, the opening at the two out-of-domain points: PointQuotients::new
// (p3-miden-lifted-fri/src/deep/interpolate.rs:81-109) and batch_eval_lifted
// (:123-201). Returns f(z_j) of every column of every matrix (in order), 4
// words per column: z_0 (c0, c1), z_1 (c0, c1). `st` keeps the point
// quotients and weights for deep_assemble, and the aligned widths.
struct DeepOpen {
    DBuf q;
    std::map<uint64_t, DBuf> weights;
    std::vector<uint64_t> aligned_w;
    uint64_t total_aligned = 0;
};
inline std::vector<uint64_t> deep_evals(Ctx &ctx, Launcher &L, const std::vector<const Mat *> &all, uint32_t lb,
                                        uint32_t log_lde, const gl::ef zs[2], uint32_t alignment, DeepOpen &st,
                                        uint64_t *d2h) {
    const TwTables &twn = ctx.twiddles(log_lde);
    const uint64_t n = 1ull << log_lde;
    const uint64_t ginv = gl::inv(gl::GEN);
    st.q = ctx.alloc(4 * n);
    DBuf &q = st.q;
    {
        deep::PQArgs a{};
        a.n = n;
        a.log_n = log_lde;
        a.wn = ntt::PowTab{twn.fwd_lo.p, twn.fwd_hi.p, twn.lo_bits};
        a.z[0] = zs[0];
        a.z[1] = zs[1];
        a.q = q.p;
        L(deep::point_quotients_kernel, blocks_for((n + deep::CHUNK - 1) / deep::CHUNK, 128), 128, 0, a);
    }
    const uint64_t d = n >> lb;
    const uint32_t log_d = log2u(d);
    std::map<uint64_t, DBuf> &weights = st.weights;
    weights[d] = ctx.alloc(4 * d);
    L(deep::top_weights_kernel, blocks_for(d, 256), 256, 0, q.p, d, log_lde,
      ntt::PowTab{twn.fwd_lo.p, twn.fwd_hi.p, twn.lo_bits}, weights[d].p);
    for (const Mat *m : all) {
        uint64_t dm = m->h >> lb;
        if (weights.count(dm)) continue;
        weights[dm] = ctx.alloc(4 * dm);
        L(deep::fold_weights_kernel, blocks_for(dm, 256), 256, 0, weights[d].p, dm, d / dm, weights[dm].p);
    }
    gl::ef sj[2];
    for (int j = 0; j < 2; j++) {
        gl::ef t = gl::ef_sub(gl::ef_exp2k(gl::ef_mulf(zs[j], ginv), log_d), gl::ef_one());
        sj[j] = gl::ef_mulf(t, gl::inv(d % gl::P));
    }
    std::vector<uint64_t> &aligned_w = st.aligned_w;
    uint64_t total_w = 0;
    for (const Mat *m : all) {
        aligned_w.push_back((m->w + alignment - 1) / alignment * alignment);
        st.total_aligned += aligned_w.back();
        total_w += m->w;
    }
    DBuf evals = ctx.alloc(4 * total_w);
    {
        uint64_t off = 0;
        for (const Mat *m : all) {
            uint64_t dm = m->h >> lb;
            uint64_t col_tiles = (m->w + 31) / 32;
            // one wave of resident blocks: as many row chunks as fit beside the
            // column tiles (a second, partial wave would double the time)
            int bps = 0, sms = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, deep::colsum_kernel, 256, 0));
            CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
            bps = std::max(1, bps);
            const uint64_t target_blocks = (uint64_t)sms * bps;
            uint64_t n_chunks = std::max<uint64_t>(1, std::min<uint64_t>(dm / 64 + 1, target_blocks / col_tiles));
            uint64_t rpc = (dm + n_chunks - 1) / n_chunks;
            n_chunks = (dm + rpc - 1) / rpc;
            DBuf part = ctx.alloc(n_chunks * m->w * 4);
            L(deep::colsum_kernel, dim3((unsigned)col_tiles, (unsigned)n_chunks), 256, 0, m->d, m->w, dm,
              weights[dm].p, rpc, part.p);
            L(deep::colsum_finish_kernel, blocks_for(m->w, 128), 128, 0, part.p, n_chunks, m->w, sj[0], sj[1],
              evals.p + 4 * off);
            off += m->w;
        }
    }
    std::vector<uint64_t> h_evals(4 * total_w);
    ctx.d2h(h_evals.data(), evals.p, 4 * total_w);
    ctx.sync();
    if (d2h) *d2h += 32 * total_w;
    return h_evals;
}

// DEEP, the quotient: DeepPoly::from_evals and accumulate_matrices
// (p3-miden-lifted-fri/src/deep/prover.rs:106-364) with the column challenge
// ac and the point challenge bp: the reduced openings f_red(z_j), coefficients
// -ac^{W-1-c} over the aligned columns, one row dot product per matrix
// (read lifted), and Q(x) = sum_j bp^j (f_red(z_j) - f_red(x)) / (z_j - x).
// Returns the n EF values of Q on the LDE domain (bit-reversed).
inline DBuf deep_assemble(Ctx &ctx, Launcher &L, const std::vector<const Mat *> &all, uint32_t log_lde,
                          const std::vector<uint64_t> &h_evals, gl::ef ac, gl::ef bp, DeepOpen &st) {
    const std::vector<uint64_t> &aligned_w_ = st.aligned_w;
    gl::ef fred[2] = {gl::ef_zero(), gl::ef_zero()};
    {
        uint64_t off = 0;
        for (size_t mi = 0; mi < all.size(); mi++) {
            for (uint64_t c = 0; c < aligned_w_[mi]; c++)
                for (int j = 0; j < 2; j++) {
                    gl::ef v = c < all[mi]->w ? gl::ef{h_evals[4 * (off + c) + 2 * j], h_evals[4 * (off + c) + 2 * j + 1]}
                                              : gl::ef_zero();
                    fred[j] = gl::ef_add(gl::ef_mul(fred[j], ac), v);
                }
            off += all[mi]->w;
        }
    }
    // coefficients -alpha^{W-1-c} over the aligned flat columns
    const uint64_t total_aligned = st.total_aligned, n = 1ull << log_lde;
    const std::vector<uint64_t> &aligned_w = st.aligned_w;
    DBuf &q = st.q;
    std::map<uint64_t, DBuf> &weights = st.weights;
    std::vector<uint64_t> coef(2 * total_aligned);
    {
        gl::ef p = gl::ef{gl::P - 1, 0};
        for (uint64_t c = total_aligned; c-- > 0;) {
            coef[2 * c] = p.c0, coef[2 * c + 1] = p.c1;
            p = gl::ef_mul(p, ac);
        }
    }
    DBuf d_coef = ctx.upload(coef);
    std::vector<DBuf> dots(all.size());
    deep::AssembleArgs aa{};
    {
        uint64_t off = 0;
        for (size_t mi = 0; mi < all.size(); mi++) {
            const Mat *m = all[mi];
            dots[mi] = ctx.alloc(2 * m->h);
            const uint64_t *cf = d_coef.p + 2 * off;
            if (m->w >= 16) {
                size_t smem = 16 * m->w;
                static std::atomic<uint64_t> attr_done{0};
                smem_attr_once(attr_done, deep::rowdot_warp_kernel, 200 * 1024);
                unsigned grid = (unsigned)std::min<uint64_t>(blocks_for(m->h * 32, 256), 148 * 16);
                L(deep::rowdot_warp_kernel, grid, 256, smem, m->d, m->h, m->w, cf, dots[mi].p);
            } else {
                L(deep::rowdot_thread_kernel, blocks_for(m->h, 256), 256, 0, m->d, m->h, m->w, cf, dots[mi].p);
            }
            aa.dots[mi] = dots[mi].p;
            aa.lift[mi] = log_lde - log2u(m->h);
            off += aligned_w[mi];
        }
    }
    aa.n_dots = (int)all.size();
    aa.q = q.p;
    aa.n = n;
    aa.fred[0] = fred[0];
    aa.fred[1] = fred[1];
    aa.beta = bp;
    DBuf layer = ctx.alloc(2 * n);
    aa.out = layer.p;
    L(deep::assemble_kernel, blocks_for(n, 256), 256, 0, aa);
    q.release();
    weights.clear();
    dots.clear();
    return layer;
}

inline void prove(Ctx &ctx, const PcsParams &pcs, const Instance *inst, size_t n_inst, ProofOut &po) {
    using clk = std::chrono::steady_clock;
    Launcher L{ctx};
    const uint32_t lb = pcs.log_blowup;
    const uint32_t log_max_h = log2u(inst[n_inst - 1].height);
    uint32_t log_qd = 0;
    for (size_t i = 0; i < n_inst; i++) log_qd = std::max(log_qd, inst_log_qd(inst[i]));
    const uint64_t D = 1ull << log_qd;
    const uint32_t log_lde = log_max_h + lb;
    const uint64_t n = 1ull << log_lde;
    Transcript tr(ctx.p2);

    cudaEvent_t ev[10];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    CK(cudaEventRecord(ev[0], ctx.stream));

    // ---- 1. main traces: coset LDE on g^(2^lift) K, bit-reversed; aligned tree
    uint64_t max_hw = 0;
    for (size_t i = 0; i < n_inst; i++)
        max_hw = std::max(max_hw, inst[i].height * std::max<uint64_t>(inst[i].width, 2 * inst_aux_width(inst[i])));
    max_hw = std::max(max_hw, inst[n_inst - 1].height * 2 * D);
    DBuf tmp = ctx.alloc(max_hw);
    std::vector<DBuf> main_lde(n_inst), aux_lde(n_inst);
    std::vector<Mat> main_mats, aux_mats;
    const uint64_t launches_before = ctx.launches;
    Tree main_tree;
    // column-major copies of the quotient-domain rows for the generated
    // constraint kernels of symbolic AIRs (main part written during the main
    // commit, aux part before the constraints), in the context's workspace
    std::vector<uint64_t *> sym_cm(n_inst, nullptr);
    {
        std::vector<uint64_t> off(n_inst, 0);
        uint64_t words = 0;
        for (size_t i = 0; i < n_inst; i++)
            if (inst[i].air == AIR_SYMBOLIC) {
                off[i] = words;
                words += (inst[i].height << inst_log_qd(inst[i])) * (inst[i].width + 2 * inst_aux_width(inst[i]));
            }
        if (words) {
            uint64_t *ws = ctx.workspace(words);
            for (size_t i = 0; i < n_inst; i++)
                if (inst[i].air == AIR_SYMBOLIC) sym_cm[i] = ws + off[i];
        }
    }
    commit_main_pipelined(ctx, inst, n_inst, lb, log_max_h, main_lde, main_mats, main_tree, po, ev[1], sym_cm);
    tr.send_commit(main_tree.root);
    CK(cudaEventRecord(ev[2], ctx.stream));

    // ---- 2. randomness (max num_randomness over the AIRs) and the aux
    // traces from each instance's AuxBuilder, EF flattened to 2 base columns
    // (prover/mod.rs:285-345). Without any builder every aux trace is zero:
    // the LDE of a zero trace on any coset is zero, and its tree has one
    // digest per layer (build_zero_tree), so both are produced exactly,
    // without transforms or per-leaf hashing.
    uint64_t n_rand = 0;
    for (size_t i = 0; i < n_inst; i++) n_rand = std::max(n_rand, inst_num_randomness(inst[i]));
    std::vector<uint64_t> rnd(2 * n_rand);
    for (uint64_t r = 0; r < n_rand; r++) {
        gl::ef e = tr.ch.sample_ef();
        rnd[2 * r] = e.c0, rnd[2 * r + 1] = e.c1;
    }
    std::vector<std::vector<uint64_t>> aux_vals(n_inst);
    bool any_builder = false;
    for (size_t i = 0; i < n_inst; i++) {
        aux_vals[i].assign(2 * inst_num_aux_values(inst[i]), 0);
        any_builder |= inst[i].aux_build != nullptr;
    }
    Tree aux_tree;
    if (!any_builder) {
        for (size_t i = 0; i < n_inst; i++) {
            const uint64_t h = inst[i].height, aw2 = 2 * inst_aux_width(inst[i]);
            aux_lde[i] = ctx.alloc((h << lb) * aw2);
            CK(cudaMemsetAsync(aux_lde[i].p, 0, (h << lb) * aw2 * 8, ctx.stream));
            aux_mats.push_back({aux_lde[i].p, h << lb, aw2});
        }
        build_zero_tree(ctx, aux_tree, aux_mats, 8);
    } else {
        for (size_t i = 0; i < n_inst; i++) {
            const Instance &I = inst[i];
            const uint64_t h = I.height, aw2 = 2 * inst_aux_width(I);
            aux_lde[i] = ctx.alloc((h << lb) * aw2);
            aux_mats.push_back({aux_lde[i].p, h << lb, aw2});
            if (!I.aux_build) {
                CK(cudaMemsetAsync(aux_lde[i].p, 0, (h << lb) * aw2 * 8, ctx.stream));
                continue;
            }
            std::vector<uint64_t> host(h * aw2, 0);
            if (I.aux_build(I.aux_user, i, I.trace, rnd.data(), inst_num_randomness(I), h, host.data(),
                            aux_vals[i].data()) != 0)
                throw CudaError{ERR_VALIDATION, "aux builder failed for instance " + std::to_string(i)};
            for (uint64_t v : host)
                if (v >= gl::P) throw CudaError{ERR_INVALID, "aux builder wrote a non-canonical word"};
            for (uint64_t v : aux_vals[i])
                if (v >= gl::P) throw CudaError{ERR_INVALID, "aux builder wrote a non-canonical aux value"};
            DBuf up = ctx.alloc(h * aw2);
            CK(cudaMemcpyAsync(up.p, host.data(), h * aw2 * 8, cudaMemcpyHostToDevice, ctx.stream));
            po.h2d += h * aw2 * 8;
            coset_lde(ctx, up.p, aw2, h, aw2, lb, gl::exp2k(gl::GEN, log_max_h - log2u(h)), aux_lde[i].p, tmp.p);
            ctx.sync();  // `host` and `up` are released at the end of this iteration
        }
        build_tree(ctx, aux_tree, aux_mats, 8);
    }
    tr.send_commit(aux_tree.root);
    for (size_t i = 0; i < n_inst; i++)  // aux values, per instance (prover/mod.rs:347-353)
        for (size_t k = 0; k < aux_vals[i].size(); k += 2) tr.send_ef(gl::ef{aux_vals[i][k], aux_vals[i][k + 1]});
    CK(cudaEventRecord(ev[3], ctx.stream));

    // ---- 4./5. alpha, beta; constraints with cyclic extension
    const gl::ef alpha = tr.ch.sample_ef();
    const gl::ef beta = tr.ch.sample_ef();
    const uint64_t max_qh = inst[n_inst - 1].height * D;
    DBuf acc = ctx.alloc(2 * max_qh);
    uint64_t acc_len = 0;
    for (size_t ii = 0; ii < n_inst; ii++) {
        const Instance &I = inst[ii];
        const uint32_t log_h = log2u(I.height);
        const uint64_t qh = I.height * D;
        const uint32_t log_qh = log_h + log_qd;
        if (acc_len == 0) {
            CK(cudaMemsetAsync(acc.p, 0, qh * 16, ctx.stream));
        } else {
            L(quot::scale_ef_kernel, blocks_for(acc_len, 256), 256, 0, acc.p, acc_len, beta);
            if (qh > acc_len) L(quot::tile_ef_kernel, blocks_for(qh - acc_len, 256), 256, 0, acc.p, acc_len, qh);
        }
        acc_len = qh;
        const uint64_t K = inst_num_constraints(I);
        std::vector<uint64_t> ap(2 * K);
        gl::ef p = gl::ef_one();
        for (uint64_t k = K; k-- > 0;) {
            ap[2 * k] = p.c0, ap[2 * k + 1] = p.c1;
            p = gl::ef_mul(p, alpha);
        }
        if (I.air == AIR_SYMBOLIC) {
            eval_symbolic(ctx, I, sym_cm[ii], aux_lde[ii].p, log_h, log_qd, log_max_h, rnd, aux_vals[ii], ap,
                          acc.p);
            L.n++;
            continue;
        }
        DBuf d_ap = ctx.upload(ap);
        DBuf d_consts;
        if (I.air == AIR_CUBIC) d_consts = ctx.upload(std::vector<uint64_t>(I.consts, I.consts + I.width));
        const TwTables &twq = ctx.twiddles(log_qh);
        quot::EvalArgs a{};
        a.lde = main_lde[ii].p;
        a.w = I.width;
        a.log_qh = log_qh;
        a.log_h = log_h;
        a.D = D;
        a.shift = gl::exp2k(gl::GEN, log_max_h - log_h);
        a.wq = ntt::PowTab{twq.fwd_lo.p, twq.fwd_hi.p, twq.lo_bits};
        a.omega_h_inv = gl::inv(gl::root(log_h));
        {
            uint64_t s_pow_n = gl::exp2k(a.shift, log_h), wd = gl::root(log_qd), x = 1;
            for (uint64_t t = 0; t < D; t++) a.zh[t] = gl::sub(gl::mul(s_pow_n, x), 1), x = gl::mul(x, wd);
        }
        a.alpha_pows = d_ap.p;
        a.consts = d_consts.p;
        a.acc = acc.p;
        if (I.air == AIR_CUBIC) L(quot::cubic_eval_kernel, blocks_for(qh * 32, 256), 256, 0, a);
        else {
            static std::atomic<uint64_t> attr_done{0};
            smem_attr_once(attr_done, quot::keccak_eval_block_kernel, (int)quot::KEC_SMEM_MAX);
            int dev_sms = 148, per_sm = 1;
            CK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx.device));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, quot::keccak_eval_block_kernel,
                                                             quot::KEC_THREADS, quot::kec_smem(D)));
            uint64_t blocks = std::min<uint64_t>(qh, (uint64_t)dev_sms * std::max(1, per_sm));
            uint64_t ppb = (qh + blocks - 1) / blocks;
            blocks = (qh + ppb - 1) / ppb;
            L(quot::keccak_eval_block_kernel, (unsigned)blocks, quot::KEC_THREADS, quot::kec_smem(D), a, ppb);
        }
        ctx.sync();  // keep d_ap / d_consts alive until the kernel ran
    }
    // ---- 6. divide by Z_H on the max quotient coset
    {
        quot::VanArgs v{};
        v.D = D;
        uint64_t s_pow_n = gl::exp2k(gl::GEN, log_max_h), wd = gl::root(log_qd), x = 1;
        for (uint64_t t = 0; t < D; t++) v.inv_van[t] = gl::inv(gl::sub(gl::mul(s_pow_n, x), 1)), x = gl::mul(x, wd);
        L(quot::divide_vanishing_kernel, blocks_for(max_qh, 256), 256, 0, acc.p, max_qh, v);
    }
    CK(cudaEventRecord(ev[4], ctx.stream));

    // ---- 7. quotient chunks: N x D EF -> (N*B) x 2D base on gK
    const uint64_t N = inst[n_inst - 1].height;
    DBuf quot_lde = ctx.alloc((N << lb) * 2 * D);
    {
        std::vector<uint64_t> col_bases(D);
        uint64_t wji = gl::inv(gl::root(log_max_h + log_qd)), x = 1;
        for (uint64_t t = 0; t < D; t++) col_bases[t] = x, x = gl::mul(x, wji);
        coset_lde(ctx, acc.p, 2 * D, N, 2 * D, lb, 1, quot_lde.p, tmp.p, col_bases);
    }
    acc.release();
    Tree quot_tree;
    build_tree(ctx, quot_tree, {{quot_lde.p, N << lb, 2 * D}}, 8);
    tr.send_commit(quot_tree.root);
    CK(cudaEventRecord(ev[5], ctx.stream));

    // ---- 8. OOD point outside H and gK (coset.rs:329-342)
    gl::ef z;
    const uint64_t ginv = gl::inv(gl::GEN);
    for (;;) {
        z = tr.ch.sample_ef();
        bool in_h = gl::ef_eq(gl::ef_exp2k(z, log_max_h), gl::ef_one());
        bool in_gk = gl::ef_eq(gl::ef_exp2k(gl::ef_mulf(z, ginv), log_lde), gl::ef_one());
        if (!in_h && !in_gk) break;
    }
    const gl::ef zs[2] = {z, gl::ef_mulf(z, gl::root(log_max_h))};

    // ---- 9. DEEP
    std::vector<const Mat *> all;
    for (auto &m : main_tree.mats) all.push_back(&m);
    for (auto &m : aux_tree.mats) all.push_back(&m);
    for (auto &m : quot_tree.mats) all.push_back(&m);
    DeepOpen dopen;
    std::vector<uint64_t> h_evals = deep_evals(ctx, L, all, lb, log_lde, zs, 8, dopen, &po.d2h);
    const std::vector<uint64_t> &aligned_w = dopen.aligned_w;
    // send aligned evals per point (deep/prover.rs:271-277)
    for (int j = 0; j < 2; j++) {
        uint64_t off = 0;
        for (size_t mi = 0; mi < all.size(); mi++) {
            for (uint64_t c = 0; c < aligned_w[mi]; c++) {
                if (c < all[mi]->w) tr.send_ef(gl::ef{h_evals[4 * (off + c) + 2 * j], h_evals[4 * (off + c) + 2 * j + 1]});
                else tr.send_ef(gl::ef_zero());
            }
            off += all[mi]->w;
        }
    }
    // grind(deep_pow_bits), then alpha (columns) and beta (points)
    auto grind = [&](uint32_t bits) {
        if (bits == 0) {
            tr.fields.push_back(0);
            return;
        }
        fri::GrindArgs g{};
        memcpy(g.state, tr.ch.state, sizeof(g.state));
        for (int i = 0; i < tr.ch.n_in; i++) g.pending[i] = tr.ch.in[i];
        g.n_pending = tr.ch.n_in;
        g.bits = bits;
        DBuf fb = ctx.alloc(1);
        uint64_t found = ~0ull;
        const uint64_t batch = 1ull << 22;
        for (uint64_t base = 0; base < (1ull << 36); base += batch) {
            CK(cudaMemsetAsync(fb.p, 0xff, 8, ctx.stream));
            g.base = base;
            g.count = batch;
            g.found = (unsigned long long *)fb.p;
            L(fri::grind_kernel, 148 * 2, 128, 0, g);
            ctx.d2h(ctx.stage(1), fb.p, 1);
            ctx.sync();
            found = ctx.pinned[0];
            if (found != ~0ull) break;
        }
        if (found == ~0ull) throw CudaError{ERR_TIMEOUT, "grind: no witness found within the search bound"};
        if (!tr.ch.check_witness(bits, found)) throw CudaError{ERR_CUDA, "grind: device witness rejected by host"};
        tr.ch.observe(found);
        (void)tr.ch.sample_bits(bits);
        tr.fields.push_back(found);
    };
    grind(pcs.deep_pow_bits);
    const gl::ef ac = tr.ch.sample_ef();
    const gl::ef bp = tr.ch.sample_ef();
    DBuf layer = deep_assemble(ctx, L, all, log_lde, h_evals, ac, bp, dopen);
    dopen = DeepOpen();
    CK(cudaEventRecord(ev[6], ctx.stream));

    // ---- FRI commit phase
    const uint32_t log_a = pcs.log_folding_arity;
    const uint64_t arity = 1ull << log_a;
    const uint32_t log_max_final = pcs.log_final_degree + lb;
    const uint64_t rounds = log_lde > log_max_final ? (log_lde - log_max_final + log_a - 1) / log_a : 0;
    const uint32_t log_final_size = log_lde - (uint32_t)rounds * log_a;
    const uint64_t final_deg = 1ull << (log_final_size > lb ? log_final_size - lb : 0);
    const uint64_t final_dom = final_deg << lb;
    const TwTables &tw0 = ctx.twiddles(log_lde);
    std::vector<DBuf> fri_layers;
    std::vector<std::unique_ptr<Tree>> fri_trees;
    uint64_t dom = n;
    fri_layers.push_back(std::move(layer));
    std::unique_ptr<Tree> next_tree;
    {
        auto t = std::make_unique<Tree>();
        if (dom > final_dom) {
            build_tree(ctx, *t, {{fri_layers[0].p, dom / arity, 2 * arity}}, 1);
            next_tree = std::move(t);
        }
    }
    uint64_t winv_a[8];
    {
        uint64_t wi = gl::inv(gl::root(log_a)), x = 1;
        for (uint64_t t = 0; t < 8; t++) winv_a[t] = x, x = gl::mul(x, wi);
    }
    // The rounds run without host round trips: the challenger lives on the
    // device for the loop (fri::DevCh). Per round: observe the root, grind,
    // check the witness and sample beta (one-thread kernels), fold + hash the
    // next round's leaves, compress. The roots, witnesses and the final
    // challenger state come back in one copy after the loop.
    const uint32_t fbits = pcs.folding_pow_bits;
    const uint64_t n_rounds = rounds;
    DBuf dch, droots, dwit, dbeta, dfound;
    if (n_rounds) {
        fri::DevCh h{};
        memcpy(h.state, tr.ch.state, sizeof(h.state));
        memcpy(h.in, tr.ch.in, sizeof(h.in));
        memcpy(h.out, tr.ch.out, sizeof(h.out));
        h.n_in = tr.ch.n_in, h.n_out = tr.ch.n_out, h.err = 0;
        dch = ctx.alloc((sizeof(fri::DevCh) + 7) / 8);
        uint64_t *st = ctx.stage((sizeof(fri::DevCh) + 7) / 8);
        memcpy(st, &h, sizeof(h));
        ctx.h2d(dch.p, st, (sizeof(fri::DevCh) + 7) / 8);
        droots = ctx.alloc(4 * n_rounds);
        dwit = ctx.alloc(n_rounds);
        dbeta = ctx.alloc(2 * n_rounds);
        dfound = ctx.alloc(n_rounds);
        CK(cudaMemsetAsync(dfound.p, 0xff, n_rounds * 8, ctx.stream));
    }
    fri::DevCh *devch = (fri::DevCh *)dch.p;
    for (uint64_t r = 0; r < n_rounds; r++) {
        Tree &cur = *next_tree;
        L(fri::fri_observe_root_kernel, 1, 32, 0, devch, (const uint64_t *)(cur.layers.p + 4 * cur.layer_off(cur.depth)),
          droots.p + 4 * r);
        fri_trees.push_back(std::move(next_tree));
        if (fbits) {
            fri::GrindArgs g{};
            g.bits = fbits;
            g.base = 0;
            g.count = 1ull << std::min<uint32_t>(40, fbits + 16);  // ~2^16 times the expected work
            g.found = (unsigned long long *)(dfound.p + r);
            g.ch = devch;
            L(fri::grind_kernel, 148 * 2, 128, 0, g);
        }
        L(fri::fri_after_grind_kernel, 1, 32, 0, devch, fbits, (const unsigned long long *)(dfound.p + r), dwit.p + r,
          dbeta.p + 2 * r);
        const uint64_t nout = dom / arity;
        DBuf out = ctx.alloc(2 * nout);
        fri::FoldArgs fa{};
        fa.in = fri_layers.back().p;
        fa.n_out = nout;
        fa.log_a = log_a;
        fa.log_nin = log2u(dom);
        fa.log_n0 = log_lde;
        fa.w0inv = ntt::PowTab{tw0.inv_lo.p, tw0.inv_hi.p, tw0.lo_bits};
        fa.beta_dev = dbeta.p + 2 * r;
        memcpy(fa.winv_a, winv_a, sizeof(winv_a));
        fa.inv_a = gl::inv(arity);
        fa.out = out.p;
        bool more = nout > final_dom;
        std::unique_ptr<Tree> nt;
        if (more) {
            nt = std::make_unique<Tree>();
            nt->mats = {{out.p, nout / arity, 2 * arity}};
            nt->alignment = 1;
            nt->H = nout / arity;
            nt->depth = log2u(nt->H);
            nt->layers = ctx.alloc((2 * nt->H - 1) * 4);
            fa.digests = nt->layers.p;
        }
        const uint64_t n_leaves = (nout + arity - 1) / arity;
        if (more && n_leaves <= 4096)  // latency-bound: one 16-lane group per leaf
            L(fri::fold_hash_coop_kernel, blocks_for(n_leaves * 16, 128), 128, 0, fa);
        else
            L(fri::fold_hash_kernel, blocks_for(n_leaves, 128), 128, 0, fa);
        if (more) {
            compress_layers(ctx, *nt);
            next_tree = std::move(nt);
        }
        fri_layers.push_back(std::move(out));
        dom = nout;
    }
    if (n_rounds) {  // the transcript entries of the loop, in order, and the challenger
        std::vector<uint64_t> roots(4 * n_rounds), wit(n_rounds);
        ctx.d2h(roots.data(), droots.p, 4 * n_rounds);
        ctx.d2h(wit.data(), dwit.p, n_rounds);
        uint64_t *st = ctx.stage((sizeof(fri::DevCh) + 7) / 8);
        ctx.d2h(st, dch.p, (sizeof(fri::DevCh) + 7) / 8);
        ctx.sync();
        fri::DevCh h;
        memcpy(&h, st, sizeof(h));
        if (h.err) throw CudaError{ERR_TIMEOUT, "FRI grind: no valid witness within the search bound"};
        for (uint64_t r = 0; r < n_rounds; r++) {
            for (int i = 0; i < 4; i++) tr.commits.push_back(roots[4 * r + i]);
            memcpy(fri_trees[r]->root, &roots[4 * r], 32);
            tr.fields.push_back(wit[r]);
        }
        memcpy(tr.ch.state, h.state, sizeof(h.state));
        memcpy(tr.ch.in, h.in, sizeof(h.in));
        memcpy(tr.ch.out, h.out, sizeof(h.out));
        tr.ch.n_in = h.n_in, tr.ch.n_out = h.n_out;
        po.d2h += 40 * n_rounds;
    }
    // final polynomial: first final_deg values, bit-reversed, iDFT, descending order
    {
        std::vector<uint64_t> last(2 * dom);
        ctx.d2h(last.data(), fri_layers.back().p, 2 * dom);
        ctx.sync();
        po.d2h += 16 * dom;
        uint32_t lf = log2u(final_deg);
        std::vector<gl::ef> v(final_deg), c(final_deg);
        for (uint64_t i = 0; i < final_deg; i++) {
            uint64_t s = gl::bitrev(i, lf);
            v[i] = gl::ef{last[2 * s], last[2 * s + 1]};
        }
        uint64_t winv = gl::inv(gl::root(lf)), finv = gl::inv(final_deg % gl::P);
        for (uint64_t k = 0; k < final_deg; k++) {
            gl::ef s = gl::ef_zero();
            for (uint64_t i = 0; i < final_deg; i++) s = gl::ef_add(s, gl::ef_mulf(v[i], gl::pow(winv, (i * k) % final_deg)));
            c[k] = gl::ef_mulf(s, finv);
        }
        for (uint64_t k = final_deg; k-- > 0;) tr.send_ef(c[k]);
    }
    CK(cudaEventRecord(ev[7], ctx.stream));

    // ---- query phase
    grind(pcs.query_pow_bits);
    std::set<uint64_t> idxset;
    for (uint32_t qi = 0; qi < pcs.num_queries; qi++) idxset.insert(gl::bitrev(tr.ch.sample_bits(log_lde), log_lde));
    std::vector<uint64_t> idx(idxset.begin(), idxset.end());
    std::vector<OpeningPlan> plans;
    std::vector<const Tree *> order = {&main_tree, &aux_tree, &quot_tree};
    for (auto *t : order) {
        plans.emplace_back();
        plan_openings(*t, idx, plans.back());
    }
    for (size_t r = 0; r < fri_trees.size(); r++) {
        std::set<uint64_t> s;
        for (uint64_t i : idx) s.insert(i >> (log_a * (r + 1)));
        plans.emplace_back();
        plan_openings(*fri_trees[r], std::vector<uint64_t>(s.begin(), s.end()), plans.back());
    }
    std::vector<Seg> segs;
    uint64_t total = 0;
    for (auto &p : plans) {
        for (auto &r : p.rows) segs.push_back({r.src, r.len, total}), total += r.len;
        for (auto *s : p.sibs) segs.push_back({s, 4, total}), total += 4;
    }
    const uint64_t *gathered = nullptr;  // pinned staging (the gathered hints)
    if (!segs.empty()) {
        DBuf d_out = ctx.alloc(total);
        std::vector<uint64_t> raw(segs.size() * 3);
        memcpy(raw.data(), segs.data(), segs.size() * sizeof(Seg));
        DBuf up = ctx.upload(raw);
        L(gather_kernel, (unsigned)std::min<size_t>(segs.size(), 65535), 128, 0, (const Seg *)up.p, (uint64_t)segs.size(),
          d_out.p);
        uint64_t *st = ctx.stage(total);
        ctx.d2h(st, d_out.p, total);
        ctx.sync();
        gathered = st;
        po.d2h += 8 * total;
    }
    {
        uint64_t n_hint_fields = 0, n_hint_commits = 0;
        for (auto &p : plans) {
            for (auto &r : p.rows) n_hint_fields += r.padded;
            n_hint_commits += 4 * p.sibs.size();
        }
        tr.fields.reserve(tr.fields.size() + n_hint_fields);
        tr.commits.reserve(tr.commits.size() + n_hint_commits);
        uint64_t off = 0;
        for (auto &p : plans) {
            for (auto &r : p.rows) {
                for (uint64_t k = 0; k < r.len; k++) tr.hint_field(gathered[off + k]);
                for (uint64_t k = r.len; k < r.padded; k++) tr.hint_field(0);
                off += r.len;
            }
            for (size_t s = 0; s < p.sibs.size(); s++) {
                tr.hint_commit(&gathered[off]);
                off += 4;
            }
        }
    }
    CK(cudaEventRecord(ev[8], ctx.stream));
    ctx.sync();
    tr.finalize(po.digest);
    for (int s = 0; s < 8; s++) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[s], ev[s + 1]));
        po.stage_ms[s] = ms;
    }  // [8] (LDE kernel time) was set by the main commit
    {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ev[0], ev[8]));
        po.stage_ms[11] = ms;  // whole proof on the device timeline
    }
    for (auto &e : ev) cudaEventDestroy(e);
    po.fields = std::move(tr.fields);
    po.commits = std::move(tr.commits);
    po.launches = L.n + ctx.launches - launches_before;
}

}  // namespace p3g
