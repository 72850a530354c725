// Verifier for the proofs of this library: verify_multi
// (p3-miden-lifted-stark/src/verifier/mod.rs:170-364) with the LMCS
// openings (p3-miden-lmcs/src/lmcs.rs:167-290), the DEEP query check
// (p3-miden-lifted-fri/src/deep/verifier.rs) and the FRI query checks
// (p3-miden-lifted-fri/src/fri/verifier.rs:113-249) on the device.
//
// The transcript replay is sequential and stays on the host: commitments,
// challenges, the out-of-domain evaluations, grinds, FRI roots and betas,
// the final polynomial and the query indices. From the indices alone the
// host then lays out every opening (rows, sibling digests, which nodes each
// compression reads), and the device does the hashing and the per-query
// arithmetic:
//  - one warp per opened leaf: the row sponge, matrix by matrix in
//    overwrite mode, on the 16-lane cooperative permutation (a Keccak row is
//    330 chained permutations, so latency decides);
//  - one launch per tree level, over all trees: compress(left, right) of
//    computed nodes and hinted siblings;
//  - one warp per query: the reduced row (a dot product with the powers of
//    the DEEP column challenge) and the DEEP quotient value;
//  - one block: the FRI rounds (position check, fold) and the final
//    polynomial.
// The out-of-domain constraint check (the quotient identity at z) is one
// extension-field evaluation; it runs on the host with the constraint bodies
// of the prover's kernels (quotient.cuh, instantiated for gl::ef).
//
// The verdict is the first failing check in verify_multi's order: shape,
// proof-of-work, trace openings (main, aux, quotient), DEEP, per FRI round
// its opening then its fold positions, final polynomial, quotient identity,
// transcript length, digest. Error kinds: VerifierError
// (verifier/mod.rs:75-98), PcsError (lifted-fri/src/verifier.rs:165),
// FriError (fri/verifier.rs:232), DeepError (deep/verifier.rs:220),
// LmcsError (lmcs/src/lib.rs:303).
#pragma once
#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <vector>

#include "context.cuh"
#include "merkle.cuh"
#include "prover.cuh"
#include "quotient.cuh"
#include "traces.cuh"
#include "transcript.cuh"

namespace p3g {
namespace vfy {

enum Verdict : int {
    ACCEPT = 0,
    V_SHAPE = 1,       // instance shapes / ConstraintDegreeTooHigh
    V_OPENING = 2,     // an opened index outside its tree
    V_ROOT = 3,        // an opening does not hash to its commitment
    V_POW = 4,         // a proof-of-work witness fails its bits
    V_DEEP = 5,        // a query point equals an out-of-domain point
    V_FRI = 6,         // a folded value does not match the next round's opening
    V_FINAL = 7,       // the final polynomial disagrees with the last fold
    V_QUOTIENT = 8,    // ConstraintMismatch at z
    V_TRANSCRIPT = 9,  // too short, or not fully consumed
    V_DIGEST = 10      // the transcript digest differs
};

// ------------------------------------------------------------ device side

struct LeafJob {
    uint64_t row_off;  // first word of the row in the rows buffer
    uint32_t w_off;    // first absorbed width in the widths table
    uint32_t n_w;      // matrices absorbed by this leaf
    uint32_t out;      // pool slot of the digest
    uint32_t pad;
};
struct CJob {
    uint32_t left, right, out;  // pool slots
};

// One warp per leaf (both 16-lane groups hash the same row, so the warp's
// shuffles stay converged whatever the row widths).
__global__ void __launch_bounds__(128) leaf_kernel(const LeafJob *jobs, uint32_t n, const uint64_t *rows,
                                                   const uint32_t *widths, uint64_t *pool) {
    __shared__ uint64_t sc[p2::N_PARAMS];
    p2x::stage_consts(sc);
    const int l = threadIdx.x & 15;
    const p2x::Lane k = p2x::lane_consts(sc, l);
    const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= n) return;  // warp-uniform
    const LeafJob job = jobs[j];
    const uint64_t *row = rows + job.row_off;
    uint64_t x = 0;
    for (uint32_t m = 0; m < job.n_w; m++) {
        const uint32_t w = widths[job.w_off + m];
        for (uint32_t i = 0; i < w; i += 8) {
            if (l < 8) x = i + l < w ? row[i + l] : 0;
            x = p2x::permute(x, l, sc, k);
        }
        row += w;
    }
    if (threadIdx.x % 32 < 4) pool[4 * (uint64_t)job.out + l] = p2w::canon(x);
}

// One warp per compression of one tree level.
__global__ void __launch_bounds__(128) compress_kernel(const CJob *jobs, uint32_t n, uint64_t *pool) {
    __shared__ uint64_t sc[p2::N_PARAMS];
    p2x::stage_consts(sc);
    const int l = threadIdx.x & 15;
    const p2x::Lane k = p2x::lane_consts(sc, l);
    const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= n) return;  // warp-uniform
    const CJob job = jobs[j];
    uint64_t x = 0;
    if (l < 4) x = pool[4 * (uint64_t)job.left + l];
    else if (l < 8) x = pool[4 * (uint64_t)job.right + l - 4];
    x = p2x::permute(x, l, sc, k);
    if (threadIdx.x % 32 < 4) pool[4 * (uint64_t)job.out + l] = p2w::canon(x);
}

struct DeepArgs {
    const uint64_t *rows;
    uint64_t goff[3], gtw[3];  // per trace group: row offset of query 0, row width
    const uint64_t *apow;      // 2 words per column: alpha_c^(T-1-i) over main|aux|quot
    const uint64_t *xq;        // query points x_q
    uint32_t nq;
    gl::ef red_open[2], zs[2], bp;
    uint64_t *de;              // out: 2 words per query
    int32_t *flags;            // flags[0]: a denominator vanished
};
// One warp per query: red_row = sum_i v_i * alpha_c^(T-1-i), then
// de = sum_p bp^p (red_open_p - red_row) / (z_p - x_q).
__global__ void __launch_bounds__(128) deep_kernel(const __grid_constant__ DeepArgs a) {
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= a.nq) return;
    gl::Acc c0, c1;
    uint64_t col = 0;
    for (int g = 0; g < 3; g++) {
        const uint64_t *row = a.rows + a.goff[g] + q * a.gtw[g];
        for (uint64_t i = lane; i < a.gtw[g]; i += 32) {
            const uint64_t v = row[i];
            c0.mac(v, a.apow[2 * (col + i)]);
            c1.mac(v, a.apow[2 * (col + i) + 1]);
        }
        col += a.gtw[g];
    }
    uint64_t r0 = c0.reduce(), r1 = c1.reduce();
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        r0 = gl::add(r0, __shfl_xor_sync(0xffffffffu, r0, off));
        r1 = gl::add(r1, __shfl_xor_sync(0xffffffffu, r1, off));
    }
    if (lane) return;
    const gl::ef red_row{r0, r1};
    gl::ef de = gl::ef_zero(), bpow = gl::ef_one();
    for (int p = 0; p < 2; p++) {
        const gl::ef den = gl::ef_sub(a.zs[p], gl::ef{a.xq[q], 0});
        if (den.c0 == 0 && den.c1 == 0) {
            a.flags[0] = 1;
            break;
        }
        de = gl::ef_add(de, gl::ef_mul(bpow, gl::ef_mul(gl::ef_sub(a.red_open[p], red_row), gl::ef_inv(den))));
        bpow = gl::ef_mul(bpow, a.bp);
    }
    a.de[2 * q] = de.c0;
    a.de[2 * q + 1] = de.c1;
}

struct FriRound {
    uint64_t row_base;      // first word of this round's opened rows (2a words per row)
    uint32_t ncur, nr;      // entries checked, rows folded
    uint32_t ent_off;       // entries in ent_k / ent_pos
    uint32_t row_off;       // rows in s_inv
    gl::ef beta;
};
struct FriArgs {
    const uint64_t *rows;
    const FriRound *rounds;
    uint32_t n_rounds, log_a;
    const uint32_t *ent_k, *ent_pos;
    const uint64_t *s_inv;
    uint64_t winv_a[8], inv_a;
    const uint64_t *de;        // round-0 values, 2 words per query
    uint64_t *cur, *nxt;       // scratch, 2 words per entry
    uint32_t n_final;          // entries after the last round
    const uint64_t *final_x;   // their points
    const uint64_t *final_poly;
    uint32_t final_deg;
    int32_t *flags;            // flags[1]: final polynomial; flags[2 + r]: round r positions
};
// One block: rounds in order, entries and rows over the threads.
__global__ void __launch_bounds__(256) fri_kernel(const __grid_constant__ FriArgs a) {
    const uint32_t A = 1u << a.log_a;
    uint64_t *cur = a.cur, *nxt = a.nxt;
    for (uint32_t i = threadIdx.x; i < (a.n_rounds ? a.rounds[0].ncur : a.n_final); i += blockDim.x)
        cur[2 * i] = a.de[2 * i], cur[2 * i + 1] = a.de[2 * i + 1];
    __syncthreads();
    for (uint32_t r = 0; r < a.n_rounds; r++) {
        const FriRound R = a.rounds[r];
        const uint64_t *rows = a.rows + R.row_base;
        for (uint32_t q = threadIdx.x; q < R.ncur; q += blockDim.x) {
            const uint64_t *row = rows + (uint64_t)a.ent_k[R.ent_off + q] * 2 * A;
            const uint32_t pos = a.ent_pos[R.ent_off + q];
            if (row[2 * pos] != cur[2 * q] || row[2 * pos + 1] != cur[2 * q + 1]) a.flags[2 + r] = 1;
        }
        for (uint32_t kk = threadIdx.x; kk < R.nr; kk += blockDim.x) {
            const uint64_t *row = rows + (uint64_t)kk * 2 * A;
            const gl::ef x = gl::ef_mulf(R.beta, a.s_inv[R.row_off + kk]);
            gl::ef res = gl::ef_zero(), xp = gl::ef_one();
            for (uint32_t j = 0; j < A; j++) {
                gl::ef u = gl::ef_zero();
                for (uint32_t t = 0; t < A; t++) {
                    const uint32_t p = gl::bitrev(t, a.log_a);
                    u = gl::ef_add(u, gl::ef_mulf(gl::ef{row[2 * p], row[2 * p + 1]}, a.winv_a[(j * t) & (A - 1)]));
                }
                res = gl::ef_add(res, gl::ef_mul(u, xp));
                xp = gl::ef_mul(xp, x);
            }
            res = gl::ef_mulf(res, a.inv_a);
            nxt[2 * kk] = res.c0, nxt[2 * kk + 1] = res.c1;
        }
        __syncthreads();
        uint64_t *t = cur;
        cur = nxt, nxt = t;
    }
    for (uint32_t q = threadIdx.x; q < a.n_final; q += blockDim.x) {
        gl::ef e = gl::ef_zero();
        for (uint32_t i = 0; i < a.final_deg; i++)
            e = gl::ef_add(gl::ef_mulf(e, a.final_x[q]), gl::ef{a.final_poly[2 * i], a.final_poly[2 * i + 1]});
        if (e.c0 != cur[2 * q] || e.c1 != cur[2 * q + 1]) a.flags[1] = 1;
    }
}

// the digests at the given pool slots, side by side
__global__ void gather_roots_kernel(const uint64_t *pool, const uint32_t *slots, uint32_t n, uint64_t *out) {
    for (uint32_t i = threadIdx.x; i < 4 * n; i += blockDim.x) out[i] = pool[4 * (uint64_t)slots[i / 4] + i % 4];
}

// -------------------------------------------------------------- host side

struct KTabHost {
    static int rot(int i) { return keccak::tables().rot[i / 5][i % 5]; }
    static uint64_t rc(int r) { return keccak::tables().rc[r]; }
};
struct EfCons {  // constraint values by index (tasks may add parts of one constraint)
    std::vector<gl::ef> v;
    void emit(int k, gl::ef x) { v[k] = gl::ef_add(v[k], x); }
};

// verify_multi's transcript reads (VerifierTranscript,
// p3-miden-transcript/src/verifier.rs): received values are observed, hints
// are not; a read past the end yields zero and marks the transcript short.
struct Reader {
    Challenger ch;
    const uint64_t *f;
    uint64_t nf, pf = 0;
    const uint64_t *c;
    uint64_t nc, pc = 0;
    bool short_read = false;
    uint64_t hint() {
        if (pf >= nf) {
            short_read = true;
            return 0;
        }
        return f[pf++];
    }
    uint64_t field() {
        if (pf >= nf) {
            short_read = true;
            return 0;
        }
        const uint64_t x = f[pf++];
        ch.observe(x);
        return x;
    }
    gl::ef ef() {
        const uint64_t a = field();
        const uint64_t b = field();
        return gl::ef{a, b};
    }
    void commit(uint64_t out[4], bool observe) {
        if (pc >= nc) {
            short_read = true;
            memset(out, 0, 32);
            return;
        }
        memcpy(out, c + 4 * pc++, 32);
        if (observe)
            for (int i = 0; i < 4; i++) ch.observe(out[i]);
    }
    // check_witness (p3-miden-transcript/src/verifier.rs): bits = 0 accepts
    // without observing the witness
    bool grind(unsigned bits) {
        const uint64_t w = hint();
        if (bits == 0) return true;
        ch.observe(w);
        return ch.sample_bits(bits) == 0;
    }
};

constexpr uint32_t kHint = 1u << 31;  // job operand tag: a hinted sibling, not a computed node

struct Batch {  // one LMCS open_batch
    uint64_t commit[4];
    uint32_t root = 0;     // node slot of the computed root
    bool bad_index = false, no_root = false;
    uint64_t row_off = 0, tw = 0;
};
struct Plan {
    std::vector<uint64_t> rows, hints;
    std::vector<uint32_t> widths;
    std::vector<LeafJob> leaves;
    std::vector<std::vector<CJob>> levels;
    std::vector<Batch> batches;
    uint32_t n_nodes = 0;

    // LMCS open_batch (lmcs.rs:167-290): rows of the sorted unique indices,
    // then siblings level by level, left to right, each streamed from the
    // proof unless the sibling is itself computed from an opened index.
    void open_batch(Reader &r, const uint64_t commit[4], const std::vector<uint32_t> &w, uint32_t log_h,
                    const std::vector<uint64_t> &idx) {
        Batch b;
        memcpy(b.commit, commit, 32);
        const uint32_t w_off = (uint32_t)widths.size();
        for (uint32_t x : w) widths.push_back(x), b.tw += x;
        b.row_off = rows.size();
        std::vector<uint64_t> pos;
        std::vector<uint32_t> id;
        for (uint64_t q : idx) {
            if (q >> log_h) {  // the reference stops at the bad index
                b.bad_index = true;
                batches.push_back(b);
                return;
            }
            const uint64_t off = rows.size();
            for (uint64_t c = 0; c < b.tw; c++) rows.push_back(r.hint());
            leaves.push_back(LeafJob{off, w_off, (uint32_t)w.size(), n_nodes, 0});
            pos.push_back(q);
            id.push_back(n_nodes++);
        }
        for (uint32_t l = 0; l < log_h; l++) {
            if (levels.size() <= l) levels.emplace_back();
            size_t np = 0, n = pos.size();
            for (size_t i = 0; i < n;) {
                const uint64_t p = pos[i];
                const uint32_t mine = id[i];
                uint32_t sib;
                if (i + 1 < n && pos[i + 1] == (p ^ 1)) {
                    sib = id[i + 1];
                    i += 2;
                } else {
                    uint64_t d[4];
                    r.commit(d, false);
                    sib = kHint | (uint32_t)(hints.size() / 4);
                    hints.insert(hints.end(), d, d + 4);
                    i += 1;
                }
                const uint32_t out = n_nodes++;
                levels[l].push_back((p & 1) ? CJob{sib, mine, out} : CJob{mine, sib, out});
                id[np] = out;
                pos[np++] = p >> 1;
            }
            pos.resize(np);
            id.resize(np);
        }
        if (pos.size() == 1 && pos[0] == 0) b.root = id[0];
        else b.no_root = true;
        batches.push_back(b);
    }
};

template <class T>
inline std::vector<uint64_t> pack(const std::vector<T> &v) {
    std::vector<uint64_t> o((v.size() * sizeof(T) + 7) / 8);
    if (!v.empty()) memcpy(o.data(), v.data(), v.size() * sizeof(T));
    return o;
}
inline std::vector<uint64_t> sort_unique(std::vector<uint64_t> v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    return v;
}

struct Timing {
    double host_ms = 0, device_ms = 0;
    uint64_t launches = 0;
};

// The folded constraints of one instance at the out-of-domain point:
// sum_k alpha^(K-1-k) C_k(L, N) with the selectors of its (lifted) domain.
inline gl::ef folded_constraints(const Instance &I, const gl::ef *L, const gl::ef *N, gl::ef first, gl::ef trans,
                                 gl::ef alpha) {
    const uint64_t w = I.width;
    gl::ef folded = gl::ef_zero();
    if (I.air == AIR_CUBIC) {
        for (uint64_t c = 0; c < w; c++) {
            const gl::ef x = L[c], y = L[c + 1 == w ? 0 : c + 1];
            const gl::ef rhs = gl::ef_add(gl::ef_add(gl::ef_mul(gl::ef_mul(x, x), x), y), gl::ef{I.consts[c], 0});
            folded = gl::ef_add(gl::ef_mul(folded, alpha), gl::ef_mul(trans, gl::ef_sub(N[c], rhs)));
        }
    } else {
        EfCons f;
        f.v.assign(air_num_constraints(AIR_KECCAK, w), gl::ef_zero());
        for (int t = 0; t < quot::KEC_TASKS; t++) quot::keccak_task<gl::ef, KTabHost>(t, L, N, first, trans, f);
        for (const gl::ef &c : f.v) folded = gl::ef_add(gl::ef_mul(folded, alpha), c);
    }
    return folded;
}

// Returns the verdict. Throws CudaError on device failures.
inline int verify(Ctx &ctx, const PcsParams &pcs, const Instance *inst, size_t n_inst, const uint64_t *fields,
                  uint64_t n_fields, const uint64_t *commits, uint64_t n_commits, const uint64_t digest[12],
                  Timing *tm) {
    const auto t0 = std::chrono::steady_clock::now();
    if (n_inst == 0 || n_inst > 8) return V_SHAPE;
    for (size_t i = 0; i < n_inst; i++)
        if (inst[i].height == 0 || (inst[i].height & (inst[i].height - 1)) || (i && inst[i].height < inst[i - 1].height))
            return V_SHAPE;
    Reader r{};
    r.ch.p2 = ctx.p2;
    r.f = fields, r.nf = n_fields, r.c = commits, r.nc = n_commits;
    const uint32_t lb = pcs.log_blowup;
    const uint32_t log_max_h = log2u(inst[n_inst - 1].height);
    uint32_t log_qd = 0;
    for (size_t i = 0; i < n_inst; i++) log_qd = std::max(log_qd, air_log_quotient_degree(inst[i].air));
    if (log_qd > lb) return V_SHAPE;
    const uint64_t D = 1ull << log_qd;
    const uint32_t log_lde = log_max_h + lb;

    // commitments and challenges in prover order
    uint64_t main_c[4], aux_c[4], quot_c[4];
    r.commit(main_c, true);
    (void)r.ch.sample_ef();  // aux randomness
    r.commit(aux_c, true);
    const gl::ef alpha = r.ch.sample_ef();
    const gl::ef beta = r.ch.sample_ef();
    r.commit(quot_c, true);
    // out-of-domain point outside H and gK (coset.rs:329-342)
    gl::ef z;
    for (;;) {
        z = r.ch.sample_ef();
        const bool in_h = gl::ef_eq(gl::ef_exp2k(z, log_max_h), gl::ef_one());
        const bool in_gk = gl::ef_eq(gl::ef_exp2k(gl::ef_mulf(z, gl::inv(gl::GEN)), log_lde), gl::ef_one());
        if (!in_h && !in_gk) break;
    }
    const gl::ef zs[2] = {z, gl::ef_mulf(z, gl::root(log_max_h))};

    // matrices: main (one per instance), aux (2 columns each), quotient (2D)
    std::vector<uint64_t> ow, aw;
    for (size_t i = 0; i < n_inst; i++) ow.push_back(inst[i].width);
    for (size_t i = 0; i < n_inst; i++) ow.push_back(2);
    ow.push_back(2 * D);
    uint64_t total_aligned = 0;
    for (uint64_t w : ow) aw.push_back((w + 7) / 8 * 8), total_aligned += aw.back();

    // DEEP oracle: aligned out-of-domain evaluations per point, grind, challenges
    std::vector<gl::ef> evals(2 * total_aligned);
    for (auto &e : evals) e = r.ef();
    bool pow_ok = r.grind(pcs.deep_pow_bits);
    const gl::ef ac = r.ch.sample_ef();
    const gl::ef bp = r.ch.sample_ef();
    gl::ef red_open[2];
    for (int p = 0; p < 2; p++) {
        gl::ef acc = gl::ef_zero();
        for (uint64_t c = 0; c < total_aligned; c++) acc = gl::ef_add(gl::ef_mul(acc, ac), evals[p * total_aligned + c]);
        red_open[p] = acc;
    }
    // FRI oracle: round commitments, grinds, betas, final polynomial
    const uint32_t log_a = pcs.log_folding_arity;
    const uint64_t arity = 1ull << log_a;
    const uint32_t log_max_final = pcs.log_final_degree + lb;
    const uint64_t rounds = log_lde > log_max_final ? (log_lde - log_max_final + log_a - 1) / log_a : 0;
    const uint32_t log_final_size = log_lde - (uint32_t)rounds * log_a;
    const uint64_t final_deg = 1ull << (log_final_size > lb ? log_final_size - lb : 0);
    std::vector<std::array<uint64_t, 4>> fri_c(rounds);
    std::vector<gl::ef> fri_beta(rounds);
    for (uint64_t rr = 0; rr < rounds; rr++) {
        r.commit(fri_c[rr].data(), true);
        pow_ok = r.grind(pcs.folding_pow_bits) && pow_ok;
        fri_beta[rr] = r.ch.sample_ef();
    }
    std::vector<uint64_t> final_poly(2 * final_deg);
    for (uint64_t i = 0; i < final_deg; i++) {
        const gl::ef e = r.ef();
        final_poly[2 * i] = e.c0, final_poly[2 * i + 1] = e.c1;
    }
    pow_ok = r.grind(pcs.query_pow_bits) && pow_ok;
    std::vector<uint64_t> idx(pcs.num_queries);
    for (auto &q : idx) q = gl::bitrev(r.ch.sample_bits(log_lde), log_lde);
    idx = sort_unique(idx);
    const uint64_t nq = idx.size();

    // openings: the three trace trees, then the FRI rounds
    Plan P;
    const uint64_t *gcommit[3] = {main_c, aux_c, quot_c};
    const size_t gfirst[4] = {0, n_inst, 2 * n_inst, 2 * n_inst + 1};
    for (int g = 0; g < 3; g++) {
        std::vector<uint32_t> w;
        for (size_t m = gfirst[g]; m < gfirst[g + 1]; m++) w.push_back((uint32_t)aw[m]);
        P.open_batch(r, gcommit[g], w, log_lde, idx);
    }
    std::vector<FriRound> fr;
    std::vector<uint32_t> ent_k, ent_pos;
    std::vector<uint64_t> s_inv;
    std::vector<uint64_t> cur_idx = idx;
    uint32_t log_dom = log_lde;
    uint64_t g_inv = gl::inv(gl::root(log_lde));
    for (uint64_t rr = 0; rr < rounds; rr++) {
        const uint32_t log_folded = log_dom - log_a;
        std::vector<uint64_t> ridx;
        for (uint64_t q : cur_idx) ridx.push_back(q >> log_a);
        ridx = sort_unique(ridx);
        FriRound R{};
        R.ncur = (uint32_t)cur_idx.size();
        R.nr = (uint32_t)ridx.size();
        R.ent_off = (uint32_t)ent_k.size();
        R.row_off = (uint32_t)s_inv.size();
        R.beta = fri_beta[rr];
        R.row_base = P.rows.size();
        P.open_batch(r, fri_c[rr].data(), {(uint32_t)(2 * arity)}, log_folded, ridx);
        for (uint64_t q : cur_idx) {
            ent_k.push_back((uint32_t)(std::lower_bound(ridx.begin(), ridx.end(), q >> log_a) - ridx.begin()));
            ent_pos.push_back((uint32_t)(q & (arity - 1)));
        }
        for (uint64_t k : ridx) s_inv.push_back(gl::pow(g_inv, gl::bitrev(k, log_folded)));
        fr.push_back(R);
        cur_idx = ridx;
        log_dom = log_folded;
        g_inv = gl::exp2k(g_inv, log_a);
    }
    std::vector<uint64_t> final_x;
    {
        const uint64_t gen = gl::root(log_dom);
        for (uint64_t q : cur_idx) final_x.push_back(gl::pow(gen, gl::bitrev(q, log_dom)));
    }
    const bool consumed = r.pf == r.nf && r.pc == r.nc;
    const bool short_read = r.short_read;
    uint64_t dg[12];
    {
        Challenger c = r.ch;
        c.duplex();
        memcpy(dg, c.state, sizeof(dg));
    }

    // quotient identity at z: one extension-field evaluation on the host,
    // run while the device kernels are in flight
    auto quotient_identity = [&]() -> bool {
        gl::ef accumulated = gl::ef_zero();
        uint64_t off = 0;
        for (size_t i = 0; i < n_inst; i++) {
            const uint32_t log_h = log2u(inst[i].height), lift = log_max_h - log_h;
            const gl::ef zl = gl::ef_exp2k(z, lift);
            const gl::ef van = gl::ef_sub(gl::ef_exp2k(zl, log_h), gl::ef_one());
            const uint64_t oinv = gl::inv(gl::root(log_h));
            const gl::ef first = gl::ef_mul(van, gl::ef_inv(gl::ef_sub(zl, gl::ef_one())));
            const gl::ef trans = gl::ef_sub(zl, gl::ef{oinv, 0});
            const gl::ef folded =
                folded_constraints(inst[i], &evals[off], &evals[total_aligned + off], first, trans, alpha);
            accumulated = gl::ef_add(gl::ef_mul(accumulated, beta), folded);
            off += aw[i];
        }
        uint64_t qoff = 0;
        for (size_t m = 0; m < 2 * n_inst; m++) qoff += aw[m];
        const gl::ef X{0, 1};
        const gl::ef u = gl::ef_exp2k(gl::ef_mulf(z, gl::inv(gl::GEN)), log_max_h);
        const uint64_t ws = gl::root(log_qd);
        uint64_t wt = 1;
        gl::ef num = gl::ef_zero(), den = gl::ef_zero();
        for (uint64_t t = 0; t < D; t++) {
            const gl::ef qt = gl::ef_add(evals[qoff + 2 * t], gl::ef_mul(X, evals[qoff + 2 * t + 1]));
            const gl::ef wgt = gl::ef_mulf(gl::ef_inv(gl::ef_sub(u, gl::ef{wt, 0})), wt);
            num = gl::ef_add(num, gl::ef_mul(wgt, qt));
            den = gl::ef_add(den, wgt);
            wt = gl::mul(wt, ws);
        }
        const gl::ef qz = gl::ef_mul(num, gl::ef_inv(den));
        const gl::ef vanish = gl::ef_sub(gl::ef_exp2k(z, log_max_h), gl::ef_one());
        return gl::ef_eq(accumulated, gl::ef_mul(qz, vanish));
    };

    // device: one upload of every input, then the leaf sponges, the tree
    // levels, the DEEP values, the FRI rounds and one read-back of the roots
    // and flags
    const uint32_t n_nodes = P.n_nodes;
    auto slot = [&](uint32_t s) { return (s & kHint) ? n_nodes + (s & ~kHint) : s; };
    std::vector<CJob> cj;
    std::vector<size_t> lv_off{0};
    for (auto &lv : P.levels) {
        for (const CJob &jb : lv) cj.push_back(CJob{slot(jb.left), slot(jb.right), jb.out});
        lv_off.push_back(cj.size());
    }
    bool trace_ok = true, fri_shape_ok = true;
    for (int g = 0; g < 3; g++) trace_ok = trace_ok && !P.batches[g].bad_index;
    for (uint64_t rr = 0; rr < rounds; rr++) fri_shape_ok = fri_shape_ok && !P.batches[3 + rr].bad_index;
    const bool run_deep = trace_ok && nq, run_fri = run_deep && fri_shape_ok;
    std::vector<uint64_t> apow, xq;
    if (run_deep) {
        apow.resize(2 * total_aligned);
        gl::ef pw = gl::ef_one();
        for (uint64_t i = total_aligned; i-- > 0;) apow[2 * i] = pw.c0, apow[2 * i + 1] = pw.c1, pw = gl::ef_mul(pw, ac);
        xq.resize(nq);
        const uint64_t gen = gl::root(log_lde);
        for (uint64_t q = 0; q < nq; q++) xq[q] = gl::mul(gl::GEN, gl::pow(gen, gl::bitrev(idx[q], log_lde)));
    }
    std::vector<uint32_t> root_slot;
    for (const Batch &B : P.batches) root_slot.push_back(B.bad_index || B.no_root ? 0 : B.root);
    struct Seg {
        const void *src;
        size_t bytes, off;
    };
    std::vector<Seg> segs;
    size_t words = 0;
    auto seg = [&](const void *src, size_t bytes) {
        segs.push_back(Seg{src, bytes, words});
        words += (bytes + 7) / 8 + 1;  // one spare word keeps every segment non-empty
        return segs.back().off;
    };
    const size_t o_rows = seg(P.rows.data(), P.rows.size() * 8);
    const size_t o_widths = seg(P.widths.data(), P.widths.size() * 4);
    const size_t o_leaves = seg(P.leaves.data(), P.leaves.size() * sizeof(LeafJob));
    const size_t o_cj = seg(cj.data(), cj.size() * sizeof(CJob));
    const size_t o_apow = seg(apow.data(), apow.size() * 8);
    const size_t o_xq = seg(xq.data(), xq.size() * 8);
    const size_t o_rounds = seg(fr.data(), fr.size() * sizeof(FriRound));
    const size_t o_ek = seg(ent_k.data(), ent_k.size() * 4);
    const size_t o_ep = seg(ent_pos.data(), ent_pos.size() * 4);
    const size_t o_sinv = seg(s_inv.data(), s_inv.size() * 8);
    const size_t o_fx = seg(final_x.data(), final_x.size() * 8);
    const size_t o_fp = seg(final_poly.data(), final_poly.size() * 8);
    const size_t o_rs = seg(root_slot.data(), root_slot.size() * 4);
    const size_t staged = words;
    const size_t o_hints = seg(P.hints.data(), P.hints.size() * 8);  // copied into the pool
    const size_t pool_words = 4 * (uint64_t)n_nodes + P.hints.size() + 4;
    const uint64_t n_flags = 2 + rounds;
    const size_t back_words = 4 * P.batches.size() + (n_flags + 1) / 2;  // roots, then flags
    const uint64_t launches0 = ctx.launches;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const auto t1 = std::chrono::steady_clock::now();
    DBuf d = ctx.alloc(staged + pool_words + 3 * (2 * nq + 2) + back_words);
    uint64_t *pool = d.p + staged, *de = pool + pool_words, *cur = de + 2 * nq + 2, *nxt = cur + 2 * nq + 2;
    uint64_t *back = nxt + 2 * nq + 2;
    uint64_t *st = ctx.stage(std::max(words, back_words));
    for (const Seg &sg : segs)
        if (sg.bytes) memcpy(st + sg.off, sg.src, sg.bytes);
    CK(cudaEventRecord(e0, ctx.stream));
    ctx.h2d(d.p, st, staged);
    ctx.h2d(pool + 4 * (uint64_t)n_nodes, st + o_hints, P.hints.size());
    CK(cudaMemsetAsync(back, 0, back_words * 8, ctx.stream));
    int32_t *d_flags = (int32_t *)(back + 4 * P.batches.size());
    if (!P.leaves.empty()) {
        const uint32_t n = (uint32_t)P.leaves.size();
        leaf_kernel<<<(n * 32 + 127) / 128, 128, 0, ctx.stream>>>((const LeafJob *)(d.p + o_leaves), n, d.p + o_rows,
                                                                  (const uint32_t *)(d.p + o_widths), pool);
        CK(cudaGetLastError());
        ctx.launches++;
    }
    for (size_t l = 0; l + 1 < lv_off.size(); l++) {
        const uint32_t n = (uint32_t)(lv_off[l + 1] - lv_off[l]);
        if (!n) continue;
        compress_kernel<<<(n * 32 + 127) / 128, 128, 0, ctx.stream>>>((const CJob *)(d.p + o_cj) + lv_off[l], n,
                                                                      pool);
        CK(cudaGetLastError());
        ctx.launches++;
    }
    if (run_deep) {
        DeepArgs da{};
        da.rows = d.p + o_rows;
        for (int g = 0; g < 3; g++) da.goff[g] = P.batches[g].row_off, da.gtw[g] = P.batches[g].tw;
        da.apow = d.p + o_apow;
        da.xq = d.p + o_xq;
        da.nq = (uint32_t)nq;
        da.red_open[0] = red_open[0], da.red_open[1] = red_open[1];
        da.zs[0] = zs[0], da.zs[1] = zs[1];
        da.bp = bp;
        da.de = de;
        da.flags = d_flags;
        deep_kernel<<<(unsigned)((nq * 32 + 127) / 128), 128, 0, ctx.stream>>>(da);
        CK(cudaGetLastError());
        ctx.launches++;
    }
    if (run_fri) {
        FriArgs fa{};
        fa.rows = d.p + o_rows;
        fa.rounds = (const FriRound *)(d.p + o_rounds);
        fa.n_rounds = (uint32_t)rounds;
        fa.log_a = log_a;
        fa.ent_k = (const uint32_t *)(d.p + o_ek);
        fa.ent_pos = (const uint32_t *)(d.p + o_ep);
        fa.s_inv = d.p + o_sinv;
        const uint64_t wi = gl::inv(gl::root(log_a));
        uint64_t x = 1;
        for (uint64_t t = 0; t < 8; t++) fa.winv_a[t] = x, x = gl::mul(x, wi);
        fa.inv_a = gl::inv(arity);
        fa.de = de;
        fa.cur = cur, fa.nxt = nxt;
        fa.n_final = (uint32_t)final_x.size();
        fa.final_x = d.p + o_fx;
        fa.final_poly = d.p + o_fp;
        fa.final_deg = (uint32_t)final_deg;
        fa.flags = d_flags;
        fri_kernel<<<1, 256, 0, ctx.stream>>>(fa);
        CK(cudaGetLastError());
        ctx.launches++;
    }
    gather_roots_kernel<<<1, 128, 0, ctx.stream>>>(pool, (const uint32_t *)(d.p + o_rs),
                                                   (uint32_t)P.batches.size(), back);
    CK(cudaGetLastError());
    ctx.launches++;
    ctx.d2h(st, back, back_words);
    CK(cudaEventRecord(e1, ctx.stream));
    const bool quotient_ok = quotient_identity();
    ctx.sync();
    std::vector<uint64_t> roots(st, st + 4 * P.batches.size());
    std::vector<int32_t> flags(n_flags);
    memcpy(flags.data(), st + 4 * P.batches.size(), n_flags * 4);
    const bool deep_bad = flags[0] != 0, final_bad = flags[1] != 0;
    float dev_ms = 0;
    CK(cudaEventElapsedTime(&dev_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (tm) {
        tm->device_ms = dev_ms;
        tm->host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        tm->launches = ctx.launches - launches0;
    }
    auto batch_err = [&](size_t b) -> int {
        const Batch &B = P.batches[b];
        if (B.bad_index) return V_OPENING;
        if (B.no_root || memcmp(roots.data() + 4 * b, B.commit, 32) != 0) return V_ROOT;
        return ACCEPT;
    };

    // the first failing check, in verify_multi's order
    if (!pow_ok) return V_POW;
    for (size_t g = 0; g < 3; g++)
        if (int e = batch_err(g)) return e;
    if (deep_bad) return V_DEEP;
    for (uint64_t rr = 0; rr < rounds; rr++) {
        if (int e = batch_err(3 + rr)) return e;
        if (flags[2 + rr]) return V_FRI;
    }
    if (final_bad) return V_FINAL;
    if (!quotient_ok) return V_QUOTIENT;
    if (short_read || !consumed) return V_TRANSCRIPT;
    if (memcmp(dg, digest, 96) != 0) return V_DIGEST;
    return ACCEPT;
}

}  // namespace vfy
}  // namespace p3g
