// Device-side generation of the Keccak-f[1600] AIR trace: the same rows as
// the host generator keccak_trace() (generate_trace_rows,
// p3-miden-lifted-examples/src/keccak.rs:54-56), written straight into HBM,
// so a caller that holds only the permutation inputs (25 words each) uploads
// those instead of the 2^log_h x 2633 trace.
//
// One block per permutation (24 rows; the last one may be truncated, and
// permutations past the inputs use the all-zero state).
//  1. Warp 0, lanes 0..24 each own lane (x, y) of the state and run the 24
//     rounds (theta column parities through shared memory, rho-pi, chi,
//     iota), recording per round: the state at the round's start, the
//     column parities C and C' = C ^ D, A' = A ^ D, A'' (chi output) and
//     A'''[0][0] (after iota).
//  2. All threads expand the records into rows: a thread decodes its
//     column's field once and writes that column of every row, so the
//     threads of a warp store consecutive columns of one row.
#pragma once
#include <cstdint>

#include "gl.cuh"

namespace tgen {

constexpr int K_STEP = 0, K_EXPORT = 24, K_PRE = 25, K_A = 125, K_C = 225, K_CP = 545, K_AP = 865, K_APP = 2465,
              K_APP00 = 2565, K_APPP00 = 2629, K_NCOLS = 2633;

__constant__ uint64_t c_rc[24];
__constant__ int c_rot[25];  // rot[x*5 + y]

struct Rec {
    uint64_t st[24][25];   // state at the round's start, lane x + 5y
    uint64_t c[24][5];     // column parities
    uint64_t cp[24][5];    // C ^ D
    uint64_t ap[24][25];   // A' = A ^ D, lane x + 5y
    uint64_t app[24][25];  // chi output, lane x + 5y
    uint64_t a3[24];       // A''[0][0] ^ RC
    uint64_t in[25];
};

__device__ __forceinline__ uint64_t rotl64(uint64_t v, int r) { return r ? (v << r) | (v >> (64 - r)) : v; }

__global__ void __launch_bounds__(128) keccak_trace_kernel(const uint64_t *inputs25, uint64_t n_perms, uint64_t h,
                                                           uint64_t *out) {
    __shared__ Rec rec;
    __shared__ uint64_t sh[25], shb[25];
    const uint64_t perm = blockIdx.x;
    const uint64_t row0 = perm * 24;
    const int nrows = (int)(h - row0 < 24 ? h - row0 : 24);
    const int tid = threadIdx.x;
    if (tid < 32) {
        const int lane = tid;
        const bool own = lane < 25;
        const int x = lane % 5, y = lane / 5;
        uint64_t v = own && perm < n_perms ? inputs25[perm * 25 + lane] : 0;
        if (own) rec.in[lane] = v;
        for (int r = 0; r < nrows; r++) {
            if (own) {
                rec.st[r][lane] = v;
                sh[lane] = v;
            }
            __syncwarp();
            uint64_t cx = 0, cxm = 0, cxp = 0;
            if (own) {
                for (int yy = 0; yy < 5; yy++) {
                    cx ^= sh[x + 5 * yy];
                    cxm ^= sh[(x + 4) % 5 + 5 * yy];
                    cxp ^= sh[(x + 1) % 5 + 5 * yy];
                }
            }
            const uint64_t d = cxm ^ rotl64(cxp, 1);
            const uint64_t ap = v ^ d;
            if (own) {
                if (y == 0) {
                    rec.c[r][x] = cx;
                    rec.cp[r][x] = cx ^ d;
                }
                rec.ap[r][lane] = ap;
                // B[y][(2x + 3y) % 5] = rotl(A'[x][y], rot[x][y]); B stored at bx + 5 by
                shb[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(ap, c_rot[x * 5 + y]);
            }
            __syncwarp();
            if (own) {
                const uint64_t app = shb[lane] ^ (~shb[(x + 1) % 5 + 5 * y] & shb[(x + 2) % 5 + 5 * y]);
                rec.app[r][lane] = app;
                v = app;
                if (lane == 0) {
                    v = app ^ c_rc[r];
                    rec.a3[r] = v;
                }
            }
            __syncwarp();
        }
    }
    __syncthreads();
    uint64_t *base = out + row0 * K_NCOLS;
    for (int col = tid; col < K_NCOLS; col += blockDim.x) {
        // decode the column once: kind, lane / index, bit or limb shift
        int kind, i = 0, sh_ = 0;
        if (col < K_EXPORT) kind = 0, i = col;
        else if (col == K_EXPORT) kind = 1;
        else if (col < K_A) kind = 2, i = (col - K_PRE) / 4, sh_ = 16 * ((col - K_PRE) % 4);
        else if (col < K_C) kind = 3, i = (col - K_A) / 4, sh_ = 16 * ((col - K_A) % 4);
        else if (col < K_CP) kind = 4, i = (col - K_C) / 64, sh_ = (col - K_C) % 64;
        else if (col < K_AP) kind = 5, i = (col - K_CP) / 64, sh_ = (col - K_CP) % 64;
        else if (col < K_APP) kind = 6, i = (col - K_AP) / 64, sh_ = (col - K_AP) % 64;
        else if (col < K_APP00) kind = 7, i = (col - K_APP) / 4, sh_ = 16 * ((col - K_APP) % 4);
        else if (col < K_APPP00) kind = 8, sh_ = col - K_APP00;
        else kind = 9, sh_ = 16 * (col - K_APPP00);
        // preimage / state / A' / A'' lanes are (y*5 + x): lane index x + 5y = i % 5 * 1 + (i / 5) * 5 = i
        for (int r = 0; r < nrows; r++) {
            uint64_t val;
            switch (kind) {
                case 0: val = i == r; break;
                case 1: val = 0; break;
                case 2: val = (rec.in[i] >> sh_) & 0xffff; break;
                case 3: val = (rec.st[r][i] >> sh_) & 0xffff; break;
                case 4: val = (rec.c[r][i] >> sh_) & 1; break;
                case 5: val = (rec.cp[r][i] >> sh_) & 1; break;
                case 6: val = (rec.ap[r][i] >> sh_) & 1; break;
                case 7: val = (rec.app[r][i] >> sh_) & 0xffff; break;
                case 8: val = (rec.app[r][0] >> sh_) & 1; break;
                default: val = (rec.a3[r] >> sh_) & 0xffff; break;
            }
            base[(uint64_t)r * K_NCOLS + col] = val;
        }
    }
}

// Forward iteration of the cubic AIR's trace (the rows after row 0):
// row r+1 = row_r^3 + rotate(row_r, 1) + k, column i of row r+1 reading
// columns i and i+1 of row r. Rows depend on each other, columns do not, so
// one block iterates one trace: thread t owns columns t, t + T, ...; row r
// sits in shared memory (two buffers), and each row is stored to HBM by
// consecutive threads (coalesced). Widths up to kCubicMaxWidth.
constexpr uint64_t kCubicMaxWidth = 8192;
__global__ void __launch_bounds__(1024) cubic_trace_kernel(const uint64_t *row0, const uint64_t *k, uint64_t w,
                                                           uint64_t h, uint64_t *out) {
    extern __shared__ uint64_t buf[];  // 2 x w
    uint64_t *cur = buf, *nxt = buf + w;
    for (uint64_t i = threadIdx.x; i < w; i += blockDim.x) {
        cur[i] = row0[i];
        out[i] = row0[i];
    }
    __syncthreads();
    for (uint64_t r = 1; r < h; r++) {
        for (uint64_t i = threadIdx.x; i < w; i += blockDim.x) {
            const uint64_t x = cur[i];
            const uint64_t v = gl::add(gl::add(gl::mul(gl::sqr(x), x), cur[i + 1 == w ? 0 : i + 1]), __ldg(k + i));
            nxt[i] = v;
            out[r * w + i] = v;
        }
        __syncthreads();
        uint64_t *t = cur;
        cur = nxt;
        nxt = t;
    }
}

}  // namespace tgen
