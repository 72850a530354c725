// FRI commit-phase kernels (p3-miden-lifted-fri/src/fri/prover.rs:190-292,
// fri/fold/arity{2,4,8}.rs) and the proof-of-work grind.
//
// Round r commits the evaluations (bit-reversed, n_r EF) as an
// (n_r/a) x 2a base matrix (EF flattened), one leaf per row, unaligned
// tree. Folding row k (the coset s*<w_a>, s = w_{n_r}^{bitrev(k)}) with
// challenge beta gives (1/a) sum_j (beta/s)^j sum_t y_t w_a^{-jt}, where the
// row holds y_t at position bitrev_{log a}(t).
//
// The fold of round r is fused with the leaf hash of round r+1: one thread
// folds a consecutive rows, stores the a folded values and hashes them as
// one leaf of the next tree.
#pragma once
#include "gl.cuh"
#include "merkle.cuh"
#include "ntt.cuh"

namespace fri {

__device__ __forceinline__ uint64_t merkle_shfl(uint64_t v, int src) { return p2x::shfl64(v, src); }

struct FoldArgs {
    const uint64_t *in;  // n_in EF
    uint64_t n_out;      // n_in / a
    uint32_t log_a;
    uint32_t log_nin;     // log2 n_in
    uint32_t log_n0;      // log2 of the root of the s_inv table
    ntt::PowTab w0inv;    // powers of w_{n0}^{-1}
    gl::ef beta;
    const uint64_t *beta_dev;  // if set, the challenge is read from here (device-side transcript)
    uint64_t winv_a[8];   // w_a^{-t}, t < a
    uint64_t inv_a;       // 1/a
    uint64_t *out;        // n_out EF
    uint64_t *digests;    // (n_out / a) digests of the next round, or null
};

__device__ __forceinline__ gl::ef fold_one(const FoldArgs &a, gl::ef beta, uint64_t k) {
    const uint32_t A = 1u << a.log_a;
    // s_inv = w_{n_in}^{-bitrev_{log n_out}(k)} = w_{n0}^{-(bitrev << (log n0 - log n_in))}
    uint64_t e = gl::bitrev(k, a.log_nin - a.log_a) << (a.log_n0 - a.log_nin);
    uint64_t s_inv = a.w0inv.at(e);
    gl::ef x = gl::ef_mulf(beta, s_inv);
    const uint64_t *row = a.in + 2 * k * A;
    if (A == 2) {
        gl::ef y0{row[0], row[1]}, y1{row[2], row[3]};
        gl::ef r = gl::ef_add(gl::ef_add(y0, y1), gl::ef_mul(gl::ef_sub(y0, y1), x));
        return gl::ef_mulf(r, a.inv_a);
    }
    gl::ef y[8];
    for (uint32_t t = 0; t < A; t++) {
        uint64_t p = gl::bitrev(t, a.log_a);
        y[t] = gl::ef{row[2 * p], row[2 * p + 1]};
    }
    gl::ef res = gl::ef_zero(), xp = gl::ef_one();
    for (uint32_t j = 0; j < A; j++) {
        gl::ef u = gl::ef_zero();
        for (uint32_t t = 0; t < A; t++) u = gl::ef_add(u, gl::ef_mulf(y[t], a.winv_a[(j * t) & (A - 1)]));
        res = gl::ef_add(res, gl::ef_mul(u, xp));
        xp = gl::ef_mul(xp, x);
    }
    return gl::ef_mulf(res, a.inv_a);
}

// thread g folds outputs [g*a, g*a + a)
__global__ void __launch_bounds__(128) fold_hash_kernel(const __grid_constant__ FoldArgs a) {
    const uint32_t A = 1u << a.log_a;
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g * A >= a.n_out) return;
    uint64_t buf[16];
    const uint32_t cnt = (uint32_t)((a.n_out - g * A) < A ? (a.n_out - g * A) : A);
    const gl::ef beta = a.beta_dev ? gl::ef{a.beta_dev[0], a.beta_dev[1]} : a.beta;
    for (uint32_t u = 0; u < cnt; u++) {
        gl::ef v = fold_one(a, beta, g * A + u);
        a.out[2 * (g * A + u)] = v.c0;
        a.out[2 * (g * A + u) + 1] = v.c1;
        buf[2 * u] = v.c0;
        buf[2 * u + 1] = v.c1;
    }
    if (a.digests && cnt == A) {
        uint64_t s[12];
#pragma unroll
        for (int i = 0; i < 12; i++) s[i] = 0;
        const uint32_t W = 2 * A;
        for (uint32_t i = 0; i < W; i += 8) {
#pragma unroll
            for (uint32_t j = 0; j < 8; j++) s[j] = (i + j < W) ? buf[i + j] : 0;
            p2_permute_dev(s);
        }
#pragma unroll
        for (int i = 0; i < 4; i++) a.digests[4 * g + i] = p2w::canon(s[i]);
    }
}

// The same fold and leaf hash with one 16-lane group per leaf, for rounds
// with few leaves (latency-bound): lane u < a folds output g*a + u, the leaf
// words (output i >> 1, component i & 1) are gathered by shuffles, and the
// group absorbs them (overwrite mode, zero-padded 8-word chunks) with the
// cooperative permutation.
__global__ void __launch_bounds__(128) fold_hash_coop_kernel(const __grid_constant__ FoldArgs a) {
    __shared__ uint64_t sc[p2::N_PARAMS];
    p2x::stage_consts(sc);
    const int l = threadIdx.x & 15;
    const p2x::Lane k = p2x::lane_consts(sc, l);
    const uint32_t A = 1u << a.log_a;
    const uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const bool ok = g * A < a.n_out;
    const uint32_t cnt = ok ? (uint32_t)((a.n_out - g * A) < A ? (a.n_out - g * A) : A) : 0;
    const gl::ef beta = a.beta_dev ? gl::ef{a.beta_dev[0], a.beta_dev[1]} : a.beta;
    uint64_t c0 = 0, c1 = 0;
    if ((uint32_t)l < cnt) {
        const gl::ef v = fold_one(a, beta, g * A + l);
        a.out[2 * (g * A + l)] = v.c0;
        a.out[2 * (g * A + l) + 1] = v.c1;
        c0 = v.c0, c1 = v.c1;
    }
    if (!a.digests) return;  // uniform over the grid
    const uint32_t W = 2 * A;
    uint64_t x = 0;
    for (uint32_t i = 0; i < W; i += 8) {
        const uint32_t idx = i + (l & 7);
        const uint64_t w0 = merkle_shfl(c0, (int)(idx >> 1) & 15), w1 = merkle_shfl(c1, (int)(idx >> 1) & 15);
        if (l < 8) x = idx < W ? ((idx & 1) ? w1 : w0) : 0;
        x = p2x::permute(x, l, sc, k);
    }
    if (cnt == A && l < 4) a.digests[4 * g + l] = p2w::canon(x);
}

// Proof-of-work search over witnesses [base, base + count): the challenger
// with `n_pending` buffered inputs observes w and samples; success when the
// sampled word (state[7] after the duplex) has its low `bits` bits zero.
// Device copy of the host Challenger (transcript.cuh) for the FRI commit
// loop: the same observe / sample / duplex rules on canonical words, so the
// state read back after the loop continues the host transcript unchanged.
struct DevCh {
    uint64_t state[12], in[8], out[8];
    int32_t n_in, n_out;
    int32_t err;  // a grind witness was missing or did not satisfy its bits
};
// Warp-cooperative challenger for the one-warp FRI kernels: the DevCh and
// the constant table are staged in shared memory (WarpChShared), both 16-lane
// groups of the warp run the duplex permutation (p2x; the second group
// duplicates the first), group 0 writes the state back and lane 0 does the
// counters. The observe / sample / duplex rules are the host Challenger's.
struct WarpChShared {
    DevCh c;
    uint64_t sc[p2::N_PARAMS];
};
struct WarpCh {
    WarpChShared &s;
    p2x::Lane k;
    int l;
    __device__ __forceinline__ WarpCh(WarpChShared &sh, const DevCh *g) : s(sh), l(threadIdx.x & 15) {
        const uint32_t *src = (const uint32_t *)g;
        uint32_t *dst = (uint32_t *)&s.c;
        for (uint32_t i = threadIdx.x; i < sizeof(DevCh) / 4; i += 32) dst[i] = src[i];
        for (int i = threadIdx.x; i < p2::N_PARAMS; i += 32) s.sc[i] = c_p2[i];
        __syncwarp();
        k = p2x::lane_consts(s.sc, l);
    }
    __device__ __forceinline__ void store(DevCh *g) {
        __syncwarp();
        const uint32_t *src = (const uint32_t *)&s.c;
        uint32_t *dst = (uint32_t *)g;
        for (uint32_t i = threadIdx.x; i < sizeof(DevCh) / 4; i += 32) dst[i] = src[i];
    }
    __device__ __forceinline__ void duplex() {
        __syncwarp();
        uint64_t x = 0;
        if (l < 12) x = l < s.c.n_in ? s.c.in[l] : s.c.state[l];
        x = p2w::canon(p2x::permute(x, l, s.sc, k));
        __syncwarp();
        if (threadIdx.x < 12) s.c.state[l] = x;
        if (threadIdx.x < 8) s.c.out[l] = x;
        if (threadIdx.x == 0) s.c.n_in = 0, s.c.n_out = 8;
        __syncwarp();
    }
    __device__ __forceinline__ void observe(uint64_t x) {
        __syncwarp();
        if (threadIdx.x == 0) s.c.n_out = 0, s.c.in[s.c.n_in++] = x;
        __syncwarp();
        if (s.c.n_in == 8) duplex();
    }
    __device__ __forceinline__ uint64_t sample() {
        __syncwarp();
        if (s.c.n_in > 0 || s.c.n_out == 0) duplex();
        const uint64_t v = s.c.out[s.c.n_out - 1];
        __syncwarp();
        if (threadIdx.x == 0) s.c.n_out--;
        __syncwarp();
        return v;
    }
};
// send_commit(root): record and observe the four root words (one warp)
__global__ void __launch_bounds__(32) fri_observe_root_kernel(DevCh *c, const uint64_t *root, uint64_t *log_root) {
    __shared__ WarpChShared sh;
    WarpCh w(sh, c);
    for (int i = 0; i < 4; i++) {
        const uint64_t x = root[i];
        if (threadIdx.x == 0) log_root[i] = x;
        w.observe(x);
    }
    w.store(c);
}
// grind(bits) with the witness found by grind_kernel, then sample the
// folding challenge beta (one warp)
__global__ void __launch_bounds__(32) fri_after_grind_kernel(DevCh *c, uint32_t bits, const unsigned long long *found,
                                                             uint64_t *log_w, uint64_t *beta_out) {
    __shared__ WarpChShared sh;
    WarpCh w(sh, c);
    if (bits == 0) {
        if (threadIdx.x == 0) *log_w = 0;
    } else {
        uint64_t x = *found;
        if (x == ~0ull) {
            if (threadIdx.x == 0) sh.c.err = 1;
            x = 0;
        }
        if (threadIdx.x == 0) *log_w = x;
        w.observe(x);
        if ((w.sample() & ((1ull << bits) - 1)) != 0 && threadIdx.x == 0) sh.c.err = 1;
    }
    const uint64_t b0 = w.sample(), b1 = w.sample();
    if (threadIdx.x == 0) beta_out[0] = b0, beta_out[1] = b1;
    w.store(c);
}

struct GrindArgs {
    uint64_t state[12];
    uint64_t pending[8];
    uint32_t n_pending;
    uint32_t bits;
    uint64_t base;
    uint64_t count;
    unsigned long long *found;  // atomicMin target, initialised to ~0
    const DevCh *ch;            // if set, state and pending inputs are read from this device challenger
};
__global__ void __launch_bounds__(128) grind_kernel(const __grid_constant__ GrindArgs a) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t mask = (1ull << a.bits) - 1;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.count; t += stride) {
        uint64_t w = a.base + t;
        if (w >= *((volatile unsigned long long *)a.found)) return;
        uint64_t s[12];
        if (a.ch) {
#pragma unroll
            for (int i = 0; i < 12; i++) s[i] = a.ch->state[i];
            const int np = a.ch->n_in;
            for (int i = 0; i < np; i++) s[i] = a.ch->in[i];
            s[np] = w;
        } else {
#pragma unroll
            for (int i = 0; i < 12; i++) s[i] = a.state[i];
            for (uint32_t i = 0; i < a.n_pending; i++) s[i] = a.pending[i];
            s[a.n_pending] = w;
        }
        p2_permute_dev(s);
        if ((p2w::canon(s[7]) & mask) == 0) atomicMin(a.found, (unsigned long long)w);
    }
}

}  // namespace fri
