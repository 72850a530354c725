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
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
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

// The same sponge with one thread per leaf, for large batches: with many
// leaves in flight throughput decides, and the single-thread permutation
// costs about a fifth of the cooperative one's issue slots.
__global__ void __launch_bounds__(128) leaf_thread_kernel(const LeafJob *jobs, uint32_t n, const uint64_t *rows,
                                                          const uint32_t *widths, uint64_t *pool) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const LeafJob job = jobs[j];
    const uint64_t *row = rows + job.row_off;
    uint64_t s[12];
#pragma unroll
    for (int i = 0; i < 12; i++) s[i] = 0;
    for (uint32_t m = 0; m < job.n_w; m++) {
        const uint32_t w = widths[job.w_off + m];
        merkle::absorb_row<false>(s, row, w, nullptr, 0);
        row += w;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) pool[4 * (uint64_t)job.out + i] = p2w::canon(s[i]);
}
constexpr uint32_t kThreadLeaves = 2048;  // from this many leaves on, one thread per leaf

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
    // `n` hinted words read in place: returns their offset in the field
    // stream. Offsets keep advancing past the end of a short stream (vpos),
    // where the device reads zeros, as the reads of hint() would give.
    uint64_t vpos = 0;
    uint64_t skip(uint64_t n) {
        if (vpos < pf) vpos = pf;  // in step with the stream until it runs out
        const uint64_t off = vpos;
        vpos += n;
        if (vpos > nf) short_read = true;
        pf = std::min(vpos, nf);
        return off;
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
    uint64_t row_off = 0, tw = 0;  // first opened row: its offset in the proof's field stream; row width
};
// Opened rows are read in place from the proof's field stream: query q's row
// of a batch starts at row_off + q * tw (rows are hinted back to back).
struct Plan {
    std::vector<uint64_t> hints;
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
        b.row_off = std::max(r.vpos, r.pf);  // where the first skip() of the batch starts
        std::vector<uint64_t> pos;
        std::vector<uint32_t> id;
        for (uint64_t q : idx) {
            if (q >> log_h) {  // the reference stops at the bad index
                b.bad_index = true;
                batches.push_back(b);
                return;
            }
            const uint64_t off = r.skip(b.tw);
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

// One proof after the host replay: the challenges, the opening layout and
// the tables of the query checks; the device pass fills roots and flags.
struct Prepared {
    int early = -1;  // a verdict known before the device pass (shape), else -1
    std::vector<Instance> inst;
    const uint64_t *fields = nullptr;  // the proof's field stream (borrowed; opened rows are read from it)
    uint64_t n_fields = 0;
    uint64_t row_end = 0;  // end of the furthest opened row (past n_fields only for a short stream)
    bool pow_ok = true, consumed = true, short_read = false, digest_ok = true;
    bool quotient_ok = false, quotient_done = false;
    uint64_t dg[12];
    gl::ef alpha, beta, z, ac, bp, red_open[2], zs[2];
    std::vector<gl::ef> evals;
    std::vector<gl::ef> rnd, auxv;  // aux randomness; aux values of every instance, in order
    std::vector<uint64_t> aw;
    uint64_t total_aligned = 0, D = 1, rounds = 0, final_deg = 1, arity = 2, nq = 0;
    uint32_t log_max_h = 0, log_qd = 0, log_lde = 0, log_a = 1;
    std::vector<uint64_t> idx, final_poly, final_x, s_inv, apow, xq;
    Plan P;
    std::vector<FriRound> fr;
    std::vector<uint32_t> ent_k, ent_pos;
    // device results
    std::vector<uint64_t> roots;
    std::vector<int32_t> flags;
};

// The quotient identity at z: one extension-field evaluation.
inline bool quotient_identity(const Prepared &v) {
    const size_t n_inst = v.inst.size();
    gl::ef accumulated = gl::ef_zero();
    uint64_t off = 0, aux_off = 0, auxv_off = 0;
    for (size_t i = 0; i < n_inst; i++) aux_off += v.aw[i];
    for (size_t i = 0; i < n_inst; i++) {
        const Instance &I = v.inst[i];
        const uint32_t log_h = log2u(I.height), lift = v.log_max_h - log_h;
        const gl::ef zl = gl::ef_exp2k(v.z, lift);
        const gl::ef van = gl::ef_sub(gl::ef_exp2k(zl, log_h), gl::ef_one());
        const uint64_t oinv = gl::inv(gl::root(log_h));
        const gl::ef first = gl::ef_mul(van, gl::ef_inv(gl::ef_sub(zl, gl::ef_one())));
        const gl::ef trans = gl::ef_sub(zl, gl::ef{oinv, 0});
        gl::ef folded;
        if (I.air == AIR_SYMBOLIC) {  // ConstraintFolder over the DAG (verifier/mod.rs:286-339)
            const sym::Desc &d = I.sym->d;
            const gl::ef X{0, 1};
            std::vector<gl::ef> al(d.aux_width), an(d.aux_width), per;
            const uint64_t T = v.total_aligned;
            for (uint32_t c = 0; c < d.aux_width; c++) {  // row_to_packed_ext
                al[c] = gl::ef_add(v.evals[aux_off + 2 * c], gl::ef_mul(X, v.evals[aux_off + 2 * c + 1]));
                an[c] = gl::ef_add(v.evals[T + aux_off + 2 * c], gl::ef_mul(X, v.evals[T + aux_off + 2 * c + 1]));
            }
            sym::periodic_at(d, 1ull << v.log_max_h, v.z, per);
            sym::Point pt{};
            pt.main_local = &v.evals[off];
            pt.main_next = &v.evals[T + off];
            pt.aux_local = al.data();
            pt.aux_next = an.data();
            pt.pub = I.pub;
            pt.rand = v.rnd.data();
            pt.auxv = v.auxv.data() + auxv_off;
            pt.periodic = per.data();
            pt.sel[0] = first;
            pt.sel[1] = gl::ef_mul(van, gl::ef_inv(gl::ef_sub(zl, gl::ef{oinv, 0})));
            pt.sel[2] = trans;
            folded = sym::fold_at(*I.sym, pt, v.alpha);
        } else {
            folded = folded_constraints(I, &v.evals[off], &v.evals[v.total_aligned + off], first, trans, v.alpha);
        }
        accumulated = gl::ef_add(gl::ef_mul(accumulated, v.beta), folded);
        off += v.aw[i];
        aux_off += v.aw[n_inst + i];
        auxv_off += inst_num_aux_values(I);
    }
    uint64_t qoff = 0;
    for (size_t m = 0; m < 2 * n_inst; m++) qoff += v.aw[m];
    const gl::ef X{0, 1};
    const gl::ef u = gl::ef_exp2k(gl::ef_mulf(v.z, gl::inv(gl::GEN)), v.log_max_h);
    const uint64_t ws = gl::root(v.log_qd);
    uint64_t wt = 1;
    gl::ef num = gl::ef_zero(), den = gl::ef_zero();
    for (uint64_t t = 0; t < v.D; t++) {
        const gl::ef qt = gl::ef_add(v.evals[qoff + 2 * t], gl::ef_mul(X, v.evals[qoff + 2 * t + 1]));
        const gl::ef wgt = gl::ef_mulf(gl::ef_inv(gl::ef_sub(u, gl::ef{wt, 0})), wt);
        num = gl::ef_add(num, gl::ef_mul(wgt, qt));
        den = gl::ef_add(den, wgt);
        wt = gl::mul(wt, ws);
    }
    const gl::ef qz = gl::ef_mul(num, gl::ef_inv(den));
    const gl::ef vanish = gl::ef_sub(gl::ef_exp2k(v.z, v.log_max_h), gl::ef_one());
    return gl::ef_eq(accumulated, gl::ef_mul(qz, vanish));
}

// Host replay of one proof (no device work; safe to run on several threads
// with distinct outputs). With `quotient` the quotient identity is checked
// here too, else by the device pass while its kernels run.
inline void prepare(const uint64_t *p2, const PcsParams &pcs, const Instance *inst, size_t n_inst,
                    const uint64_t *fields, uint64_t n_fields, const uint64_t *commits, uint64_t n_commits,
                    const uint64_t digest[12], bool quotient, Prepared &v) {
    v.inst.assign(inst, inst + n_inst);
    v.fields = fields, v.n_fields = n_fields;
    if (n_inst == 0 || n_inst > 8) {
        v.early = V_SHAPE;
        return;
    }
    for (size_t i = 0; i < n_inst; i++)
        if (inst[i].height == 0 || (inst[i].height & (inst[i].height - 1)) || (i && inst[i].height < inst[i - 1].height)) {
            v.early = V_SHAPE;
            return;
        }
    Reader r{};
    r.ch.p2 = p2;
    r.f = fields, r.nf = n_fields, r.c = commits, r.nc = n_commits;
    const uint32_t lb = pcs.log_blowup;
    v.log_max_h = log2u(inst[n_inst - 1].height);
    uint64_t n_rand = 0, n_auxv = 0;
    for (size_t i = 0; i < n_inst; i++) {
        v.log_qd = std::max(v.log_qd, inst_log_qd(inst[i]));
        n_rand = std::max(n_rand, inst_num_randomness(inst[i]));
        n_auxv += inst_num_aux_values(inst[i]);
    }
    if (v.log_qd > lb) {
        v.early = V_SHAPE;
        return;
    }
    v.D = 1ull << v.log_qd;
    v.log_lde = v.log_max_h + lb;
    const uint32_t log_lde = v.log_lde;

    // commitments and challenges in prover order
    uint64_t main_c[4], aux_c[4], quot_c[4];
    r.commit(main_c, true);
    v.rnd.resize(n_rand);
    for (auto &e : v.rnd) e = r.ch.sample_ef();  // aux randomness
    r.commit(aux_c, true);
    v.auxv.resize(n_auxv);
    for (auto &e : v.auxv) e = r.ef();  // aux values (verifier/mod.rs:230-239)
    v.alpha = r.ch.sample_ef();
    v.beta = r.ch.sample_ef();
    r.commit(quot_c, true);
    // out-of-domain point outside H and gK (coset.rs:329-342)
    for (;;) {
        v.z = r.ch.sample_ef();
        const bool in_h = gl::ef_eq(gl::ef_exp2k(v.z, v.log_max_h), gl::ef_one());
        const bool in_gk = gl::ef_eq(gl::ef_exp2k(gl::ef_mulf(v.z, gl::inv(gl::GEN)), log_lde), gl::ef_one());
        if (!in_h && !in_gk) break;
    }
    v.zs[0] = v.z;
    v.zs[1] = gl::ef_mulf(v.z, gl::root(v.log_max_h));

    // matrices: main (one per instance), aux (2 columns each), quotient (2D)
    std::vector<uint64_t> ow;
    for (size_t i = 0; i < n_inst; i++) ow.push_back(inst[i].width);
    for (size_t i = 0; i < n_inst; i++) ow.push_back(2 * inst_aux_width(inst[i]));
    ow.push_back(2 * v.D);
    for (uint64_t w : ow) v.aw.push_back((w + 7) / 8 * 8), v.total_aligned += v.aw.back();
    const uint64_t T = v.total_aligned;

    // DEEP oracle: aligned out-of-domain evaluations per point, grind, challenges
    v.evals.resize(2 * T);
    for (auto &e : v.evals) e = r.ef();
    v.pow_ok = r.grind(pcs.deep_pow_bits);
    v.ac = r.ch.sample_ef();
    v.bp = r.ch.sample_ef();
    for (int p = 0; p < 2; p++) {
        gl::ef acc = gl::ef_zero();
        for (uint64_t c = 0; c < T; c++) acc = gl::ef_add(gl::ef_mul(acc, v.ac), v.evals[p * T + c]);
        v.red_open[p] = acc;
    }
    // FRI oracle: round commitments, grinds, betas, final polynomial
    v.log_a = pcs.log_folding_arity;
    v.arity = 1ull << v.log_a;
    const uint32_t log_max_final = pcs.log_final_degree + lb;
    v.rounds = log_lde > log_max_final ? (log_lde - log_max_final + v.log_a - 1) / v.log_a : 0;
    const uint32_t log_final_size = log_lde - (uint32_t)v.rounds * v.log_a;
    v.final_deg = 1ull << (log_final_size > lb ? log_final_size - lb : 0);
    std::vector<std::array<uint64_t, 4>> fri_c(v.rounds);
    std::vector<gl::ef> fri_beta(v.rounds);
    for (uint64_t rr = 0; rr < v.rounds; rr++) {
        r.commit(fri_c[rr].data(), true);
        v.pow_ok = r.grind(pcs.folding_pow_bits) && v.pow_ok;
        fri_beta[rr] = r.ch.sample_ef();
    }
    v.final_poly.resize(2 * v.final_deg);
    for (uint64_t i = 0; i < v.final_deg; i++) {
        const gl::ef e = r.ef();
        v.final_poly[2 * i] = e.c0, v.final_poly[2 * i + 1] = e.c1;
    }
    v.pow_ok = r.grind(pcs.query_pow_bits) && v.pow_ok;
    v.idx.resize(pcs.num_queries);
    for (auto &q : v.idx) q = gl::bitrev(r.ch.sample_bits(log_lde), log_lde);
    v.idx = sort_unique(v.idx);
    v.nq = v.idx.size();

    // openings: the three trace trees, then the FRI rounds
    const uint64_t *gcommit[3] = {main_c, aux_c, quot_c};
    const size_t gfirst[4] = {0, n_inst, 2 * n_inst, 2 * n_inst + 1};
    for (int g = 0; g < 3; g++) {
        std::vector<uint32_t> w;
        for (size_t m = gfirst[g]; m < gfirst[g + 1]; m++) w.push_back((uint32_t)v.aw[m]);
        v.P.open_batch(r, gcommit[g], w, log_lde, v.idx);
    }
    std::vector<uint64_t> cur_idx = v.idx;
    uint32_t log_dom = log_lde;
    uint64_t g_inv = gl::inv(gl::root(log_lde));
    for (uint64_t rr = 0; rr < v.rounds; rr++) {
        const uint32_t log_folded = log_dom - v.log_a;
        std::vector<uint64_t> ridx;
        for (uint64_t q : cur_idx) ridx.push_back(q >> v.log_a);
        ridx = sort_unique(ridx);
        FriRound R{};
        R.ncur = (uint32_t)cur_idx.size();
        R.nr = (uint32_t)ridx.size();
        R.ent_off = (uint32_t)v.ent_k.size();
        R.row_off = (uint32_t)v.s_inv.size();
        R.beta = fri_beta[rr];
        R.row_base = std::max(r.vpos, r.pf);
        v.P.open_batch(r, fri_c[rr].data(), {(uint32_t)(2 * v.arity)}, log_folded, ridx);
        for (uint64_t q : cur_idx) {
            v.ent_k.push_back((uint32_t)(std::lower_bound(ridx.begin(), ridx.end(), q >> v.log_a) - ridx.begin()));
            v.ent_pos.push_back((uint32_t)(q & (v.arity - 1)));
        }
        for (uint64_t k : ridx) v.s_inv.push_back(gl::pow(g_inv, gl::bitrev(k, log_folded)));
        v.fr.push_back(R);
        cur_idx = ridx;
        log_dom = log_folded;
        g_inv = gl::exp2k(g_inv, v.log_a);
    }
    {
        const uint64_t gen = gl::root(log_dom);
        for (uint64_t q : cur_idx) v.final_x.push_back(gl::pow(gen, gl::bitrev(q, log_dom)));
    }
    v.consumed = r.pf == r.nf && r.pc == r.nc;
    v.row_end = std::max(r.vpos, r.pf);
    v.short_read = r.short_read;
    {
        Challenger c = r.ch;
        c.duplex();
        memcpy(v.dg, c.state, sizeof(v.dg));
        v.digest_ok = memcmp(v.dg, digest, 96) == 0;
    }
    // tables of the DEEP check
    v.apow.resize(2 * T);
    gl::ef pw = gl::ef_one();
    for (uint64_t i = T; i-- > 0;) v.apow[2 * i] = pw.c0, v.apow[2 * i + 1] = pw.c1, pw = gl::ef_mul(pw, v.ac);
    v.xq.resize(v.nq);
    const uint64_t gen = gl::root(log_lde);
    for (uint64_t q = 0; q < v.nq; q++) v.xq[q] = gl::mul(gl::GEN, gl::pow(gen, gl::bitrev(v.idx[q], log_lde)));
    if (quotient) v.quotient_ok = quotient_identity(v), v.quotient_done = true;
}

// The device pass over several prepared proofs: one staged upload, the leaf
// sponges of every proof in one launch, every tree level of every proof in
// one launch per level, then per proof the DEEP and FRI kernels, and one
// read-back of all roots and flags. Proofs decided early are skipped.
inline void device_pass(Ctx &ctx, const std::vector<Prepared *> &vs, Timing *tm, unsigned threads = 1) {
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
    std::vector<Prepared *> act;
    for (Prepared *v : vs)
        if (v->early < 0) act.push_back(v);
    const size_t nj = act.size();
    // per proof: offsets into the shared rows / widths / nodes / hints
    std::vector<uint64_t> row_base(nj), node_base(nj), hint_base(nj), flag_base(nj), root_base(nj);
    uint64_t n_rows = 0, n_nodes = 0, n_hints = 0, n_flags = 0, n_roots = 0;
    uint32_t n_widths = 0;
    for (size_t j = 0; j < nj; j++) {
        const Plan &P = act[j]->P;
        row_base[j] = n_rows, node_base[j] = n_nodes, hint_base[j] = n_hints / 4;
        flag_base[j] = n_flags, root_base[j] = n_roots;
        n_rows += std::max(act[j]->row_end, act[j]->n_fields) + 1;  // the field stream, then zeros
        n_nodes += P.n_nodes, n_hints += P.hints.size(), n_widths += P.widths.size();
        n_flags += 2 + act[j]->rounds;
        n_roots += P.batches.size();
    }
    std::vector<uint32_t> widths, root_slot;
    std::vector<uint64_t> hints;
    std::vector<LeafJob> leaves;
    std::vector<std::vector<CJob>> levels;
    widths.reserve(n_widths), hints.reserve(n_hints);
    for (size_t j = 0; j < nj; j++) {
        const Plan &P = act[j]->P;
        const uint32_t w0 = (uint32_t)widths.size();
        widths.insert(widths.end(), P.widths.begin(), P.widths.end());
        hints.insert(hints.end(), P.hints.begin(), P.hints.end());
        auto slot = [&](uint32_t s) {
            return (s & kHint) ? (uint32_t)(n_nodes + hint_base[j] + (s & ~kHint)) : (uint32_t)(node_base[j] + s);
        };
        for (const LeafJob &L : P.leaves)
            leaves.push_back(LeafJob{row_base[j] + L.row_off, w0 + L.w_off, L.n_w, (uint32_t)(node_base[j] + L.out), 0});
        if (levels.size() < P.levels.size()) levels.resize(P.levels.size());
        for (size_t l = 0; l < P.levels.size(); l++)
            for (const CJob &c : P.levels[l]) levels[l].push_back(CJob{slot(c.left), slot(c.right), slot(c.out)});
        for (const Batch &B : P.batches) root_slot.push_back(B.bad_index || B.no_root ? 0 : slot(B.root));
    }
    std::vector<CJob> cj;
    std::vector<size_t> lv_off{0};
    for (auto &lv : levels) {
        cj.insert(cj.end(), lv.begin(), lv.end());
        lv_off.push_back(cj.size());
    }
    const size_t o_rows = seg(nullptr, n_rows * 8);  // filled from each proof's field stream below
    const size_t o_widths = seg(widths.data(), widths.size() * 4);
    const size_t o_leaves = seg(leaves.data(), leaves.size() * sizeof(LeafJob));
    const size_t o_cj = seg(cj.data(), cj.size() * sizeof(CJob));
    const size_t o_rs = seg(root_slot.data(), root_slot.size() * 4);
    std::vector<size_t> o_apow(nj), o_xq(nj), o_rounds(nj), o_ek(nj), o_ep(nj), o_sinv(nj), o_fx(nj), o_fp(nj);
    std::vector<std::vector<FriRound>> frs(nj);  // rounds with row offsets into the shared rows
    for (size_t j = 0; j < nj; j++) {
        const Prepared &v = *act[j];
        o_apow[j] = seg(v.apow.data(), v.apow.size() * 8);
        o_xq[j] = seg(v.xq.data(), v.xq.size() * 8);
        frs[j] = v.fr;
        for (FriRound &R : frs[j]) R.row_base += row_base[j];
        o_rounds[j] = seg(frs[j].data(), frs[j].size() * sizeof(FriRound));
        o_ek[j] = seg(v.ent_k.data(), v.ent_k.size() * 4);
        o_ep[j] = seg(v.ent_pos.data(), v.ent_pos.size() * 4);
        o_sinv[j] = seg(v.s_inv.data(), v.s_inv.size() * 8);
        o_fx[j] = seg(v.final_x.data(), v.final_x.size() * 8);
        o_fp[j] = seg(v.final_poly.data(), v.final_poly.size() * 8);
    }
    const size_t staged = words;
    const size_t o_hints = seg(hints.data(), hints.size() * 8);  // copied into the pool
    const size_t pool_words = 4 * n_nodes + hints.size() + 4;
    uint64_t max_nq = 0;
    for (Prepared *v : act) max_nq = std::max(max_nq, v->nq);
    const size_t q_words = 2 * max_nq + 2;
    const size_t back_words = 4 * n_roots + (n_flags + 1) / 2;  // roots, then flags
    const uint64_t launches0 = ctx.launches;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    DBuf d = ctx.alloc(staged + pool_words + 3 * q_words * std::max<size_t>(nj, 1) + back_words);
    uint64_t *pool = d.p + staged, *qbuf = pool + pool_words, *back = qbuf + 3 * q_words * std::max<size_t>(nj, 1);
    uint64_t *st = ctx.stage(std::max(words, back_words));
    for (const Seg &sg : segs)
        if (sg.bytes && sg.src) memcpy(st + sg.off, sg.src, sg.bytes);
    {  // each proof's field stream into its region, on up to `threads` host threads
        std::atomic<size_t> next{0};
        auto copy = [&]() {
            for (size_t j; (j = next.fetch_add(1)) < nj;) {
                uint64_t *dst = st + o_rows + row_base[j];
                const uint64_t nf = act[j]->n_fields;
                if (nf) memcpy(dst, act[j]->fields, nf * 8);
                memset(dst + nf, 0, (std::max(act[j]->row_end, nf) + 1 - nf) * 8);
            }
        };
        std::vector<std::thread> th;
        for (unsigned t = 1; t < std::min<size_t>(threads, nj); t++) th.emplace_back(copy);
        copy();
        for (auto &t : th) t.join();
    }
    CK(cudaEventRecord(e0, ctx.stream));
    ctx.h2d(d.p, st, staged);
    ctx.h2d(pool + 4 * n_nodes, st + o_hints, hints.size());
    CK(cudaMemsetAsync(back, 0, back_words * 8, ctx.stream));
    int32_t *d_flags = (int32_t *)(back + 4 * n_roots);
    if (!leaves.empty()) {
        const uint32_t n = (uint32_t)leaves.size();
        if (n >= kThreadLeaves)
            leaf_thread_kernel<<<(n + 127) / 128, 128, 0, ctx.stream>>>((const LeafJob *)(d.p + o_leaves), n,
                                                                        d.p + o_rows, (const uint32_t *)(d.p + o_widths),
                                                                        pool);
        else
            leaf_kernel<<<(n * 32 + 127) / 128, 128, 0, ctx.stream>>>((const LeafJob *)(d.p + o_leaves), n,
                                                                      d.p + o_rows, (const uint32_t *)(d.p + o_widths),
                                                                      pool);
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
    for (size_t j = 0; j < nj; j++) {
        const Prepared &v = *act[j];
        const Plan &P = v.P;
        bool trace_ok = true, fri_shape_ok = true;
        for (int g = 0; g < 3; g++) trace_ok = trace_ok && !P.batches[g].bad_index;
        for (uint64_t rr = 0; rr < v.rounds; rr++) fri_shape_ok = fri_shape_ok && !P.batches[3 + rr].bad_index;
        if (!trace_ok || !v.nq) continue;
        uint64_t *de = qbuf + 3 * q_words * j, *cur = de + q_words, *nxt = cur + q_words;
        int32_t *fl = d_flags + flag_base[j];
        DeepArgs da{};
        da.rows = d.p + o_rows;
        for (int g = 0; g < 3; g++) da.goff[g] = row_base[j] + P.batches[g].row_off, da.gtw[g] = P.batches[g].tw;
        da.apow = d.p + o_apow[j];
        da.xq = d.p + o_xq[j];
        da.nq = (uint32_t)v.nq;
        da.red_open[0] = v.red_open[0], da.red_open[1] = v.red_open[1];
        da.zs[0] = v.zs[0], da.zs[1] = v.zs[1];
        da.bp = v.bp;
        da.de = de;
        da.flags = fl;
        deep_kernel<<<(unsigned)((v.nq * 32 + 127) / 128), 128, 0, ctx.stream>>>(da);
        CK(cudaGetLastError());
        ctx.launches++;
        if (!fri_shape_ok) continue;
        FriArgs fa{};
        fa.rows = d.p + o_rows;
        fa.rounds = (const FriRound *)(d.p + o_rounds[j]);
        fa.n_rounds = (uint32_t)v.rounds;
        fa.log_a = v.log_a;
        fa.ent_k = (const uint32_t *)(d.p + o_ek[j]);
        fa.ent_pos = (const uint32_t *)(d.p + o_ep[j]);
        fa.s_inv = d.p + o_sinv[j];
        const uint64_t wi = gl::inv(gl::root(v.log_a));
        uint64_t x = 1;
        for (uint64_t t = 0; t < 8; t++) fa.winv_a[t] = x, x = gl::mul(x, wi);
        fa.inv_a = gl::inv(v.arity);
        fa.de = de;
        fa.cur = cur, fa.nxt = nxt;
        fa.n_final = (uint32_t)v.final_x.size();
        fa.final_x = d.p + o_fx[j];
        fa.final_poly = d.p + o_fp[j];
        fa.final_deg = (uint32_t)v.final_deg;
        fa.flags = fl;
        fri_kernel<<<1, 256, 0, ctx.stream>>>(fa);
        CK(cudaGetLastError());
        ctx.launches++;
    }
    if (n_roots) {
        gather_roots_kernel<<<1, 128, 0, ctx.stream>>>(pool, (const uint32_t *)(d.p + o_rs), (uint32_t)n_roots, back);
        CK(cudaGetLastError());
        ctx.launches++;
    }
    ctx.d2h(st, back, back_words);
    CK(cudaEventRecord(e1, ctx.stream));
    for (Prepared *v : act)
        if (!v->quotient_done) v->quotient_ok = quotient_identity(*v), v->quotient_done = true;
    ctx.sync();
    for (size_t j = 0; j < nj; j++) {
        Prepared &v = *act[j];
        v.roots.assign(st + 4 * root_base[j], st + 4 * (root_base[j] + v.P.batches.size()));
        v.flags.resize(2 + v.rounds);
        memcpy(v.flags.data(), (const int32_t *)(st + 4 * n_roots) + flag_base[j], v.flags.size() * 4);
    }
    float dev_ms = 0;
    CK(cudaEventElapsedTime(&dev_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (tm) tm->device_ms = dev_ms, tm->launches = ctx.launches - launches0;
}

// Lmcs::open_batch (p3-miden-lmcs/src/lmcs.rs:167-290) on the device: the
// hinted rows of each sorted unique index (absorbed widths, the salt last for
// a hiding tree), then the streamed siblings, hashed to a root and compared
// with the commitment. Returns ACCEPT, V_OPENING (an index outside the tree),
// V_ROOT, or V_TRANSCRIPT (hints too short or not all used).
inline int lmcs_open_batch(Ctx &ctx, const uint64_t commit[4], const std::vector<uint32_t> &widths, uint32_t log_h,
                           const std::vector<uint64_t> &idx, const uint64_t *fields, uint64_t n_fields,
                           const uint64_t *commits, uint64_t n_commits) {
    Reader r{};
    r.ch.p2 = ctx.p2;
    r.f = fields, r.nf = n_fields, r.c = commits, r.nc = n_commits;
    Plan P;
    P.open_batch(r, commit, widths, log_h, idx);
    const Batch &B = P.batches[0];
    if (B.bad_index) return V_OPENING;
    const uint64_t row_end = std::max(r.vpos, r.pf);
    const uint32_t n_nodes = P.n_nodes;
    auto slot = [&](uint32_t s) { return (s & kHint) ? n_nodes + (s & ~kHint) : s; };
    std::vector<CJob> cj;
    std::vector<size_t> lv_off{0};
    for (auto &lv : P.levels) {
        for (const CJob &c : lv) cj.push_back(CJob{slot(c.left), slot(c.right), c.out});
        lv_off.push_back(cj.size());
    }
    const uint64_t rows_w = std::max(row_end, n_fields) + 1;
    const uint64_t o_widths = rows_w, o_leaves = o_widths + (P.widths.size() + 1) / 2 + 1;
    const uint64_t o_cj = o_leaves + P.leaves.size() * sizeof(LeafJob) / 8 + 1;
    const uint64_t o_pool = o_cj + (cj.size() * sizeof(CJob) + 7) / 8 + 1;
    const uint64_t total = o_pool + 4 * (uint64_t)n_nodes + P.hints.size() + 4;
    DBuf d = ctx.alloc(total);
    uint64_t *st = ctx.stage(total);
    memset(st, 0, o_pool * 8);
    if (n_fields) memcpy(st, fields, n_fields * 8);
    memcpy(st + o_widths, P.widths.data(), P.widths.size() * 4);
    memcpy(st + o_leaves, P.leaves.data(), P.leaves.size() * sizeof(LeafJob));
    memcpy(st + o_cj, cj.data(), cj.size() * sizeof(CJob));
    memcpy(st + o_pool + 4 * (uint64_t)n_nodes, P.hints.data(), P.hints.size() * 8);
    ctx.h2d(d.p, st, total);
    uint64_t *pool = d.p + o_pool;
    if (!P.leaves.empty()) {
        const uint32_t n = (uint32_t)P.leaves.size();
        leaf_kernel<<<(n * 32 + 127) / 128, 128, 0, ctx.stream>>>((const LeafJob *)(d.p + o_leaves), n, d.p,
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
    uint64_t root[4] = {0, 0, 0, 0};
    if (!B.no_root) {
        ctx.d2h(st, pool + 4 * (uint64_t)B.root, 4);
        ctx.sync();
        memcpy(root, st, 32);
    }
    if (B.no_root || memcmp(root, commit, 32) != 0) return V_ROOT;
    if (r.short_read || r.pf != r.nf || r.pc != r.nc) return V_TRANSCRIPT;
    return ACCEPT;
}

// The first failing check, in verify_multi's order.
inline int verdict(const Prepared &v) {
    if (v.early >= 0) return v.early;
    const Plan &P = v.P;
    auto batch_err = [&](size_t b) -> int {
        const Batch &B = P.batches[b];
        if (B.bad_index) return V_OPENING;
        if (B.no_root || memcmp(v.roots.data() + 4 * b, B.commit, 32) != 0) return V_ROOT;
        return ACCEPT;
    };
    if (!v.pow_ok) return V_POW;
    for (size_t g = 0; g < 3; g++)
        if (int e = batch_err(g)) return e;
    if (v.flags[0]) return V_DEEP;
    for (uint64_t rr = 0; rr < v.rounds; rr++) {
        if (int e = batch_err(3 + rr)) return e;
        if (v.flags[2 + rr]) return V_FRI;
    }
    if (v.flags[1]) return V_FINAL;
    if (!v.quotient_ok) return V_QUOTIENT;
    if (v.short_read || !v.consumed) return V_TRANSCRIPT;
    if (!v.digest_ok) return V_DIGEST;
    return ACCEPT;
}

// One proof. Throws CudaError on device failures.
inline int verify(Ctx &ctx, const PcsParams &pcs, const Instance *inst, size_t n_inst, const uint64_t *fields,
                  uint64_t n_fields, const uint64_t *commits, uint64_t n_commits, const uint64_t digest[12],
                  Timing *tm) {
    const auto t0 = std::chrono::steady_clock::now();
    Prepared v;
    prepare(ctx.p2, pcs, inst, n_inst, fields, n_fields, commits, n_commits, digest, false, v);
    const auto t1 = std::chrono::steady_clock::now();
    if (tm) tm->host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (v.early >= 0) return v.early;
    device_pass(ctx, {&v}, tm);
    return verdict(v);
}

struct ProofRef {  // one proof of a batch
    PcsParams pcs;
    const Instance *inst;
    size_t n_inst;
    const uint64_t *fields;
    uint64_t n_fields;
    const uint64_t *commits;
    uint64_t n_commits;
    const uint64_t *digest;
};
// Several proofs: the host replays run on up to `threads` host threads
// (each with its quotient identity), then one device pass serves them all.
inline void verify_batch(Ctx &ctx, const std::vector<ProofRef> &ps, unsigned threads, int *verdicts, Timing *tm) {
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<Prepared> vs(ps.size());
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < ps.size();) {
            const ProofRef &p = ps[i];
            prepare(ctx.p2, p.pcs, p.inst, p.n_inst, p.fields, p.n_fields, p.commits, p.n_commits, p.digest, true,
                    vs[i]);
        }
    };
    threads = std::max(1u, std::min<unsigned>(threads, (unsigned)ps.size()));
    std::vector<std::thread> th;
    for (unsigned t = 1; t < threads; t++) th.emplace_back(work);
    work();
    for (auto &t : th) t.join();
    const auto t1 = std::chrono::steady_clock::now();
    if (tm) tm->host_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    std::vector<Prepared *> ptrs;
    for (auto &v : vs) ptrs.push_back(&v);
    device_pass(ctx, ptrs, tm, threads);
    for (size_t i = 0; i < vs.size(); i++) verdicts[i] = verdict(vs[i]);
}

}  // namespace vfy
}  // namespace p3g
