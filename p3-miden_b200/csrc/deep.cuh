// DEEP quotient kernels (p3-miden-lifted-fri/src/deep/{interpolate,prover}.rs).
//
//  q[i][j] = 1 / (z_j - x_i) for the bit-reversed coset points
//  x_i = g * w_n^{bitrev(i)} of gK, j in {0, 1}: chunked Montgomery batch
//  inversion (one EF inversion per CHUNK points per thread).
//
//  OOD evaluation of a committed matrix of LDE height h_m (trace degree
//  d_m = h_m / B) at z_j^{n/h_m}: f = s_j * sum_{i < d_m} W_{d_m}[i][j] * M[i],
//  with W_d[i][j] = x_i q[i][j] for the top degree and smaller degrees folded
//  by summing consecutive blocks (interpolate.rs:123-201).
//
//  DEEP polynomial: Q(x_i) = sum_j beta^j q[i][j] (f_red(z_j) - f_red(x_i))
//  with f_red(x_i) = sum_m dot(coef_m, M_m[i >> lift_m])
//  (deep/prover.rs:304-405).
#pragma once
#include "gl.cuh"
#include "ntt.cuh"

namespace deep {

constexpr int CHUNK = 8;

struct PQArgs {
    uint64_t n;
    uint32_t log_n;
    ntt::PowTab wn;  // powers of w_n
    gl::ef z[2];
    uint64_t *q;  // n x 2 EF
};

__global__ void __launch_bounds__(128) point_quotients_kernel(const __grid_constant__ PQArgs a) {
    const uint64_t i0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * CHUNK;
    if (i0 >= a.n) return;
    const int cnt = (int)((a.n - i0) < (uint64_t)CHUNK ? (a.n - i0) : (uint64_t)CHUNK);
    gl::ef d[2 * CHUNK], pre[2 * CHUNK];
    gl::ef run = gl::ef_one();
    for (int t = 0; t < cnt; t++) {
        uint64_t x = gl::mul(gl::GEN, a.wn.at(gl::bitrev(i0 + t, a.log_n)));
        for (int j = 0; j < 2; j++) {
            d[2 * t + j] = gl::ef_sub(a.z[j], gl::ef{x, 0});
            pre[2 * t + j] = run;
            run = gl::ef_mul(run, d[2 * t + j]);
        }
    }
    gl::ef inv = gl::ef_inv(run);
    for (int t = cnt - 1; t >= 0; t--)
        for (int j = 1; j >= 0; j--) {
            gl::ef r = gl::ef_mul(inv, pre[2 * t + j]);
            inv = gl::ef_mul(inv, d[2 * t + j]);
            uint64_t *o = a.q + 4 * (i0 + t) + 2 * j;
            o[0] = r.c0;
            o[1] = r.c1;
        }
}

// W[i][j] = x_i * q[i][j] for i < d
__global__ void top_weights_kernel(const uint64_t *q, uint64_t d, uint32_t log_n, ntt::PowTab wn, uint64_t *W) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d) return;
    uint64_t x = gl::mul(gl::GEN, wn.at(gl::bitrev(i, log_n)));
#pragma unroll
    for (int k = 0; k < 4; k++) W[4 * i + k] = gl::mul(q[4 * i + k], x);
}
// Wsmall[i] = sum_{c < r} Wbig[i*r + c]
__global__ void fold_weights_kernel(const uint64_t *Wb, uint64_t n_small, uint64_t r, uint64_t *Ws) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_small) return;
    uint64_t s[4] = {0, 0, 0, 0};
    for (uint64_t c = 0; c < r; c++)
#pragma unroll
        for (int k = 0; k < 4; k++) s[k] = gl::add(s[k], Wb[4 * (i * r + c) + k]);
#pragma unroll
    for (int k = 0; k < 4; k++) Ws[4 * i + k] = s[k];
}

// Column sums: partial[chunk][col][0..4) = sum over rows of chunk of
// W[i][j] * M[i][col] (EF for j = 0, 1). Block: 32 columns x 8 row lanes.
__global__ void __launch_bounds__(256) colsum_kernel(const uint64_t *M, uint64_t w, uint64_t d, const uint64_t *W,
                                                     uint64_t rows_per_chunk, uint64_t *partial) {
    __shared__ uint64_t red[8][32][4];
    const int cl = threadIdx.x & 31, rl = threadIdx.x >> 5;
    // grid: x = column tile (fastest), y = row chunk
    const uint64_t col = (uint64_t)blockIdx.x * 32 + cl;
    const uint64_t r0 = (uint64_t)blockIdx.y * rows_per_chunk;
    const uint64_t r1 = min(d, r0 + rows_per_chunk);
    gl::Acc acc[4];
    if (col < w) {
        // four rows per step: their loads are issued together, so that each
        // thread keeps several DRAM reads in flight
        uint64_t i = r0 + rl;
        for (; i + 24 < r1; i += 32) {
            uint64_t v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) v[u] = __ldg(M + (i + 8 * u) * w + col);
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int k = 0; k < 4; k++) acc[k].mac(v[u], __ldg(W + 4 * (i + 8 * u) + k));
        }
        for (; i < r1; i += 8) {
            uint64_t v = __ldg(M + i * w + col);
#pragma unroll
            for (int k = 0; k < 4; k++) acc[k].mac(v, __ldg(W + 4 * i + k));
        }
    }
    uint64_t s[4];
#pragma unroll
    for (int k = 0; k < 4; k++) red[rl][cl][k] = s[k] = acc[k].reduce();
    __syncthreads();
    if (rl == 0 && col < w) {
        for (int r = 1; r < 8; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) s[k] = gl::add(s[k], red[r][cl][k]);
#pragma unroll
        for (int k = 0; k < 4; k++) partial[(blockIdx.y * w + col) * 4 + k] = s[k];
    }
}
// out[col][0..4) = s_j * sum_chunk partial[chunk][col]
__global__ void colsum_finish_kernel(const uint64_t *partial, uint64_t n_chunks, uint64_t w, gl::ef s0, gl::ef s1,
                                     uint64_t *out) {
    uint64_t col = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= w) return;
    uint64_t s[4] = {0, 0, 0, 0};
    for (uint64_t c = 0; c < n_chunks; c++)
#pragma unroll
        for (int k = 0; k < 4; k++) s[k] = gl::add(s[k], partial[(c * w + col) * 4 + k]);
    gl::ef e0 = gl::ef_mul(gl::ef{s[0], s[1]}, s0), e1 = gl::ef_mul(gl::ef{s[2], s[3]}, s1);
    out[4 * col + 0] = e0.c0;
    out[4 * col + 1] = e0.c1;
    out[4 * col + 2] = e1.c0;
    out[4 * col + 3] = e1.c1;
}

// Row dot products dots[i] = sum_col coef[col] * M[i][col] (EF coef).
// Wide matrices: one warp per row, coefficients staged in shared memory.
__global__ void __launch_bounds__(256) rowdot_warp_kernel(const uint64_t *M, uint64_t h, uint64_t w,
                                                          const uint64_t *coef, uint64_t *dots) {
    extern __shared__ uint64_t sc[];
    for (uint64_t k = threadIdx.x; k < 2 * w; k += blockDim.x) sc[k] = coef[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < h; i += warps) {
        const uint64_t *row = M + i * w;
        gl::Acc a0, a1;
        uint64_t col = lane;
        for (; col + 96 < w; col += 128) {  // four loads in flight per lane
            uint64_t v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) v[u] = __ldg(row + col + 32 * u);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                a0.mac(v[u], sc[2 * (col + 32 * u)]);
                a1.mac(v[u], sc[2 * (col + 32 * u) + 1]);
            }
        }
        for (; col < w; col += 32) {
            uint64_t v = __ldg(row + col);
            a0.mac(v, sc[2 * col]);
            a1.mac(v, sc[2 * col + 1]);
        }
        uint64_t c0 = a0.reduce(), c1 = a1.reduce();
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            c0 = gl::add(c0, __shfl_xor_sync(0xffffffffu, c0, off));
            c1 = gl::add(c1, __shfl_xor_sync(0xffffffffu, c1, off));
        }
        if (lane == 0) {
            dots[2 * i] = c0;
            dots[2 * i + 1] = c1;
        }
    }
}
// Narrow matrices: one thread per row.
__global__ void rowdot_thread_kernel(const uint64_t *M, uint64_t h, uint64_t w, const uint64_t *coef, uint64_t *dots) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= h) return;
    const uint64_t *row = M + i * w;
    gl::Acc a0, a1;
    for (uint64_t col = 0; col < w; col++) {
        uint64_t v = __ldg(row + col);
        a0.mac(v, __ldg(coef + 2 * col));
        a1.mac(v, __ldg(coef + 2 * col + 1));
    }
    dots[2 * i] = a0.reduce();
    dots[2 * i + 1] = a1.reduce();
}

constexpr int MAX_DOTS = 24;
struct AssembleArgs {
    const uint64_t *dots[MAX_DOTS];
    uint32_t lift[MAX_DOTS];
    int n_dots;
    const uint64_t *q;
    uint64_t n;
    gl::ef fred[2];
    gl::ef beta;
    uint64_t *out;  // n EF
};
__global__ void __launch_bounds__(256) assemble_kernel(const __grid_constant__ AssembleArgs a) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    gl::ef negf = gl::ef_zero();
    for (int m = 0; m < a.n_dots; m++) {
        const uint64_t *d = a.dots[m] + 2 * (i >> a.lift[m]);
        negf = gl::ef_add(negf, gl::ef{__ldg(d), __ldg(d + 1)});
    }
    const uint64_t *q = a.q + 4 * i;
    gl::ef r = gl::ef_mul(gl::ef{q[0], q[1]}, gl::ef_add(a.fred[0], negf));
    gl::ef r1 = gl::ef_mul(gl::ef{q[2], q[3]}, gl::ef_add(a.fred[1], negf));
    r = gl::ef_add(r, gl::ef_mul(a.beta, r1));
    a.out[2 * i] = r.c0;
    a.out[2 * i + 1] = r.c1;
}

}  // namespace deep
