// Batched two-adic NTTs over row-major Goldilocks matrices and the
// bit-reversed coset LDE built from them.
//
// A matrix is h x w, row-major, one polynomial per column. A pass loads a
// group of G = 2^k rows (stride 2^blo) for a tile of C columns into shared
// memory, runs k radix-2 stages on it and stores it back; a transform of
// size 2^L is ceil(L/10) passes. Rows are C*8 contiguous bytes per tile, so
// any row permutation (bit reversal on load) is free at that granularity.
//
// Coset LDE of a trace on s*K, |K| = h*B (used for traces, aux traces and
// quotient chunks):
//   1. inverse transform, DIT: rows read at bit-reversed positions, output
//      natural-order coefficients (times h);
//   2. for each of the B cosets (s*w_{hB}^k)*H of K: scale coefficient i by
//      (s*w_{hB}^k)^i / h and run a forward DIF transform of size h; DIF
//      leaves its output in bit-reversed order, which is exactly the
//      committed layout: coset k occupies rows [bitrev_B(k)*h, +h) of the
//      bit-reversed LDE.
#pragma once
#include "gl.cuh"

namespace ntt {

// Two-level power table: v^e = hi[e >> lo_bits] * lo[e & (2^lo_bits - 1)].
struct PowTab {
    const uint64_t *lo;
    const uint64_t *hi;
    uint32_t lo_bits;
    __device__ __forceinline__ uint64_t at(uint64_t e) const {
        uint64_t a = __ldg(lo + (e & ((1ull << lo_bits) - 1)));
        uint64_t eh = e >> lo_bits;
        return eh ? gl::mul(a, __ldg(hi + eh)) : a;
    }
};

struct PassArgs {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t ld_src, ld_dst;  // row strides in elements
    uint64_t w;               // columns
    uint32_t L;               // log2 of transform size
    uint32_t blo, bhi;        // bit range handled by this pass (bhi - blo <= 10)
    uint32_t src_bitrev;      // 1: element p is read from source row bitrev_L(p)
    PowTab tw;                // powers of the transform root w_n (forward or inverse)
    const uint64_t *tw1024;   // w_1024^j (same direction), j < 512
    uint32_t has_scale;       // multiply loaded element at natural index i by scale.at(i)
    PowTab scale;
};

// Twiddle of the butterfly on global bit b = blo + q for in-group index m:
//   w_n^{(i mod 2^b) << (L-1-b)} = w_n^{base_lo << (L-1-b)} * w_{2^{q+1}}^{m mod 2^q}
// The second factor is the size-2^(q+1) root, read from a shared table of
// w_1024 powers; the first is one constant per (block, stage), 1 when the
// pass starts at bit 0.
template <int C, bool DIF>
__global__ void __launch_bounds__(256) ntt_pass_kernel(const __grid_constant__ PassArgs a) {
    extern __shared__ uint64_t sm[];
    const uint32_t k = a.bhi - a.blo;
    const uint32_t G = 1u << k;
    uint64_t *tw = sm + (size_t)G * C;  // 512 entries
    uint64_t *sc = tw + 512;            // per-stage constants, indexed by q
    const uint64_t S = 1ull << a.blo;
    const uint64_t g = blockIdx.x;
    const uint64_t base = (g & (S - 1)) | ((g >> a.blo) << a.bhi);
    const uint64_t base_lo = base & (S - 1);
    const uint64_t col0 = (uint64_t)blockIdx.y * C;
    const int tid = threadIdx.x;
    const int c = tid % C;
    const int rstep = blockDim.x / C;
    const bool col_ok = col0 + c < a.w;
    for (uint32_t m = tid / C; m < G; m += rstep) {
        uint64_t i = base + (uint64_t)m * S;
        uint64_t row = a.src_bitrev ? gl::bitrev(i, a.L) : i;
        uint64_t v = col_ok ? __ldg(a.src + row * a.ld_src + col0 + c) : 0;
        if (a.has_scale) v = gl::mul(v, a.scale.at(i));
        sm[m * C + c] = v;
    }
    for (uint32_t t = tid; t < 512; t += blockDim.x) tw[t] = __ldg(a.tw1024 + t);
    if (tid < (int)k) sc[tid] = base_lo ? a.tw.at(base_lo << (a.L - 1 - (a.blo + tid))) : 1;
    __syncthreads();
    const uint32_t nbf = G / 2;
    for (uint32_t st = 0; st < k; st++) {
        const uint32_t q = DIF ? (k - 1 - st) : st;
        const uint32_t half = 1u << q;
        const uint64_t cst = sc[q];
        for (uint32_t j = tid / C; j < nbf; j += rstep) {
            const uint32_t jl = j & (half - 1);
            const uint32_t m = ((j >> q) << (q + 1)) | jl;
            uint64_t w = tw[jl << (9 - q)];
            if (base_lo) w = gl::mul(w, cst);
            uint64_t u = sm[m * C + c], v = sm[(m + half) * C + c];
            if (DIF) {
                sm[m * C + c] = gl::add(u, v);
                sm[(m + half) * C + c] = gl::mul(gl::sub(u, v), w);
            } else {
                uint64_t tv = gl::mul(v, w);
                sm[m * C + c] = gl::add(u, tv);
                sm[(m + half) * C + c] = gl::sub(u, tv);
            }
        }
        __syncthreads();
    }
    if (!col_ok) return;
    for (uint32_t m = tid / C; m < G; m += rstep) {
        uint64_t i = base + (uint64_t)m * S;
        a.dst[i * a.ld_dst + col0 + c] = sm[m * C + c];
    }
}

// Radix-8 register variant (k >= 3 bits per pass). Each thread owns 8
// elements of one column per round and runs 3 stages in registers; the
// shared-memory tile is touched once per round instead of once per stage.
// Twiddles of every in-group stage q, including the per-block constant of
// strided passes, are precomputed per block into T_q[x] = cst_q * w_{2^{q+1}}^x
// (x < 2^q, stored at offset 2^q - 1), so a butterfly costs one table load.
template <int C, bool DIF>
__global__ void __launch_bounds__(1024) ntt_pass_r8_kernel(const __grid_constant__ PassArgs a) {
    extern __shared__ uint64_t sm[];
    const uint32_t k = a.bhi - a.blo;
    const uint32_t G = 1u << k;
    const uint32_t TPC = G >> 3;  // threads per column
    uint64_t *tq = sm + (size_t)G * C;  // G - 1 twiddles
    uint64_t *sc = tq + G;              // per-stage constants
    const uint64_t S = 1ull << a.blo;
    // grid: x = column tile (fastest), y = row group, so that blocks resident
    // at the same time read and write whole rows
    const uint64_t g = blockIdx.y;
    const uint64_t base = (g & (S - 1)) | ((g >> a.blo) << a.bhi);
    const uint64_t base_lo = base & (S - 1);
    const uint64_t col0 = (uint64_t)blockIdx.x * C;
    const uint32_t tid = threadIdx.x;
    const uint32_t c = tid % C, t = tid / C;
    const bool col_ok = col0 + c < a.w;
    // load 8 elements (rows t + i*TPC)
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t m = t + i * TPC;
        uint64_t gi = base + (uint64_t)m * S;
        uint64_t row = a.src_bitrev ? gl::bitrev(gi, a.L) : gi;
        uint64_t v = col_ok ? __ldg(a.src + row * a.ld_src + col0 + c) : 0;
        if (a.has_scale) v = gl::mul(v, a.scale.at(gi));
        sm[m * C + c] = v;
    }
    for (uint32_t q = tid; q < k; q += blockDim.x) sc[q] = base_lo ? a.tw.at(base_lo << (a.L - 1 - (a.blo + q))) : 1;
    __syncthreads();
    for (uint32_t idx = tid; idx < G - 1; idx += blockDim.x) {
        uint32_t q = 31 - __clz(idx + 1);
        uint32_t x = idx + 1 - (1u << q);
        uint64_t w = __ldg(a.tw1024 + (x << (9 - q)));
        tq[idx] = base_lo ? gl::mul(w, sc[q]) : w;
    }
    __syncthreads();
    // rounds of up to 3 bits; DIF walks bits downwards, DIT upwards
    const uint32_t nr = (k + 2) / 3;
    for (uint32_t rd = 0; rd < nr; rd++) {
        uint32_t q_lo, r;
        if (DIF) {
            int hi = (int)k - 3 * (int)rd;
            q_lo = hi >= 3 ? hi - 3 : 0;
            r = hi - q_lo;
        } else {
            q_lo = 3 * rd;
            r = k - q_lo < 3 ? k - q_lo : 3;
        }
        const uint32_t E = 1u << r;         // elements per task
        const uint32_t tasks = G >> r;      // tasks per column
        for (uint32_t task = t; task < tasks; task += TPC) {
            const uint32_t low = task & ((1u << q_lo) - 1);
            const uint32_t high = task >> q_lo;
            const uint32_t mb = low | (high << (q_lo + r));
            uint64_t x[8];
#pragma unroll
            for (uint32_t j = 0; j < 8; j++)
                if (j < E) x[j] = sm[(mb | (j << q_lo)) * C + c];
            if (DIF) {
#pragma unroll
                for (int s = 2; s >= 0; s--) {
                    if ((uint32_t)s >= r) continue;
                    const uint32_t q = q_lo + s, hs = 1u << s;
                    const uint64_t *T = tq + (1u << q) - 1;
#pragma unroll
                    for (uint32_t j = 0; j < 8; j++) {
                        if (j >= E || (j & hs)) continue;
                        uint64_t w = T[low + ((j & (hs - 1)) << q_lo)];
                        uint64_t u = x[j], v = x[j + hs];
                        x[j] = gl::add(u, v);
                        x[j + hs] = gl::mul(gl::sub(u, v), w);
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < 3; s++) {
                    if ((uint32_t)s >= r) continue;
                    const uint32_t q = q_lo + s, hs = 1u << s;
                    const uint64_t *T = tq + (1u << q) - 1;
#pragma unroll
                    for (uint32_t j = 0; j < 8; j++) {
                        if (j >= E || (j & hs)) continue;
                        uint64_t w = T[low + ((j & (hs - 1)) << q_lo)];
                        uint64_t u = x[j], v = gl::mul(x[j + hs], w);
                        x[j] = gl::add(u, v);
                        x[j + hs] = gl::sub(u, v);
                    }
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < 8; j++)
                if (j < E) sm[(mb | (j << q_lo)) * C + c] = x[j];
        }
        __syncthreads();
    }
    if (!col_ok) return;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        uint32_t m = t + i * TPC;
        uint64_t gi = base + (uint64_t)m * S;
        a.dst[gi * a.ld_dst + col0 + c] = sm[m * C + c];
    }
}

// Multiply row k, column col of a row-major matrix by col_base[col/2]^k
// (quotient chunk de-shifting, quotient.rs:484-497). col_base holds one
// value per EF column.
static __global__ void scale_rows_by_colpow_kernel(uint64_t *m, uint64_t h, uint64_t w, const uint64_t *col_base_pows_lo,
                                            const uint64_t *col_base_pows_hi, uint32_t lo_bits, uint64_t hi_len) {
    uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= h * w) return;
    uint64_t r = idx / w, col = idx % w, t = col / 2;
    uint64_t lo = col_base_pows_lo[t * (1ull << lo_bits) + (r & ((1ull << lo_bits) - 1))];
    uint64_t hi = col_base_pows_hi[t * hi_len + (r >> lo_bits)];
    m[idx] = gl::mul(m[idx], gl::mul(lo, hi));
}

}  // namespace ntt
