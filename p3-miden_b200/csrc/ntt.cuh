// Two-level power tables, and the radix-2 shared-memory NTT pass used by
// the allocation-free LDE entry point (the prover's LDE kernels are in
// lde.cuh).
//
// A matrix is h x w, row-major, one polynomial per column. A pass loads a
// group of G = 2^k rows (stride 2^blo) for a tile of C columns into shared
// memory, runs k radix-2 stages on it and stores it back; a transform of
// size 2^L is ceil(L/10) passes. The coset LDE built from these passes is
// the same computation as lde.cuh's: inverse transform (DIT, rows read at
// bit-reversed positions), then per coset c the scale (s*w_{hB}^c)^i / h
// and a forward DIF transform whose bit-reversed output is the coset's
// block of the committed layout.
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

}  // namespace ntt
