// Quotient-numerator kernels: AIR constraint evaluation on the quotient
// coset gJ, alpha-folding, beta/cyclic accumulation across traces and the
// vanishing-polynomial division.
//
// For a trace of height h committed on the (lifted) coset s*K, gJ is the
// prefix of h*D rows of its bit-reversed LDE: natural point m of gJ
// (x_m = s * w_{hD}^m) sits at LDE row bitrev_{log hD}(m), and the "next"
// row is point (m + D) mod hD (prover/commit.rs:134-144,
// constraints/mod.rs:117-128). The folded numerator is
// sum_k alpha^{K-1-k} C_k(x_m) (constraints/mod.rs:50-56); alpha^{K-1-k} is
// precomputed per constraint, so the fold is a dot product.
#pragma once
#include "gl.cuh"
#include "ntt.cuh"

namespace quot {

struct EvalArgs {
    const uint64_t *lde;  // bit-reversed LDE of the trace, row stride w
    uint64_t w;
    uint32_t log_qh;       // log2(h * D)
    uint32_t log_h;
    uint64_t D;
    uint64_t shift;        // coset shift s of this trace
    ntt::PowTab wq;        // powers of w_{hD}
    uint64_t omega_h_inv;  // w_h^{-1}
    uint64_t zh[8];        // Z_H(x) = x^h - 1 on gJ, periodic with period D
    const uint64_t *alpha_pows;  // 2 words per constraint: alpha^{K-1-k}
    const uint64_t *consts;      // AIR constants (cubic: k[w])
    uint64_t *acc;               // EF accumulator, 2 words per point
};

struct Fold {
    uint64_t c0 = 0, c1 = 0;
    const uint64_t *ap;
    int k = 0;
    __device__ __forceinline__ explicit Fold(const uint64_t *a) : ap(a) {}
    __device__ __forceinline__ void emit(uint64_t v) {
        uint64_t a0 = __ldg(ap + 2 * k), a1 = __ldg(ap + 2 * k + 1);
        c0 = gl::add(c0, gl::mul(v, a0));
        c1 = gl::add(c1, gl::mul(v, a1));
        k++;
    }
};

__device__ __forceinline__ uint64_t point_x(const EvalArgs &a, uint64_t m) { return gl::mul(a.shift, a.wq.at(m)); }

// ---------------------------------------------------------------- cubic
// Constraint i = is_transition * (next[i] - (local[i]^3 + local[(i+1)%w] + k_i));
// the common factor is_transition is applied once per point.
// One warp per point, lanes over columns.
__global__ void __launch_bounds__(256) cubic_eval_kernel(const __grid_constant__ EvalArgs a) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint64_t qh = 1ull << a.log_qh;
    if (warp >= qh) return;
    const uint64_t m = warp;
    const uint64_t *L = a.lde + gl::bitrev(m, a.log_qh) * a.w;
    const uint64_t *N = a.lde + gl::bitrev((m + a.D) & (qh - 1), a.log_qh) * a.w;
    gl::Acc a0, a1;
    for (uint64_t i = lane; i < a.w; i += 32) {
        uint64_t x = __ldg(L + i);
        uint64_t y = __ldg(L + (i + 1 == a.w ? 0 : i + 1));
        uint64_t rhs = gl::add(gl::add(gl::mul(gl::sqr(x), x), y), __ldg(a.consts + i));
        uint64_t v = gl::sub(__ldg(N + i), rhs);
        a0.mac(v, __ldg(a.alpha_pows + 2 * i));
        a1.mac(v, __ldg(a.alpha_pows + 2 * i + 1));
    }
    uint64_t c0 = a0.reduce(), c1 = a1.reduce();
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        c0 = gl::add(c0, __shfl_xor_sync(0xffffffffu, c0, off));
        c1 = gl::add(c1, __shfl_xor_sync(0xffffffffu, c1, off));
    }
    if (lane == 0) {
        uint64_t trans = gl::sub(point_x(a, m), a.omega_h_inv);
        uint64_t *o = a.acc + 2 * m;
        o[0] = gl::add(o[0], gl::mul(c0, trans));
        o[1] = gl::add(o[1], gl::mul(c1, trans));
    }
}

// --------------------------------------------------------------- keccak
// Column layout of the Keccak-f[1600] AIR (2633 columns).
constexpr int KC_STEP = 0, KC_EXPORT = 24, KC_PRE = 25, KC_A = 125, KC_C = 225, KC_CP = 545, KC_AP = 865,
              KC_APP = 2465, KC_APP00 = 2565, KC_APPP00 = 2629, KC_NCOLS = 2633;

__constant__ uint64_t c_keccak_rc[24];
__constant__ int c_keccak_rot[25];  // rot[x*5+y]

// The constraint bodies are generic over the value type: base-field words
// (the prover's LDE rows, on the device) and extension elements (the
// verifier's out-of-domain rows, on the host). fo:: overloads resolve at
// compile time, so the base-field instance is the plain gl:: arithmetic.
namespace fo {
GL_HD uint64_t add(uint64_t a, uint64_t b) { return gl::add(a, b); }
GL_HD gl::ef add(gl::ef a, gl::ef b) { return gl::ef_add(a, b); }
GL_HD uint64_t sub(uint64_t a, uint64_t b) { return gl::sub(a, b); }
GL_HD gl::ef sub(gl::ef a, gl::ef b) { return gl::ef_sub(a, b); }
GL_HD uint64_t mul(uint64_t a, uint64_t b) { return gl::mul(a, b); }
GL_HD gl::ef mul(gl::ef a, gl::ef b) { return gl::ef_mul(a, b); }
GL_HD uint64_t dbl(uint64_t a) { return gl::dbl(a); }
GL_HD gl::ef dbl(gl::ef a) { return gl::ef_add(a, a); }
GL_HD uint64_t mulc(uint64_t a, uint64_t c) { return gl::mul(a, c); }  // by a base-field constant
// a product that goes straight into the fold: the lazy accumulator takes any
// 64-bit word, so the device form skips the final canonicalisation
GL_HD uint64_t mulw(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return gl::mul_weak(a, b);
#else
    return gl::mul(a, b);
#endif
}
GL_HD gl::ef mulw(gl::ef a, gl::ef b) { return gl::ef_mul(a, b); }
GL_HD gl::ef mulc(gl::ef a, uint64_t c) { return gl::ef_mulf(a, c); }
GL_HD void konst(uint64_t c, uint64_t &out) { out = c; }
GL_HD void konst(uint64_t c, gl::ef &out) { out = gl::ef{c, 0}; }
template <class T>
GL_HD T k(uint64_t c) {
    T v;
    konst(c, v);
    return v;
}
}  // namespace fo

template <class T>
GL_HD T kxor2(T a, T b) { return fo::sub(fo::add(a, b), fo::dbl(fo::mul(a, b))); }
template <class T>
GL_HD T kxor3(T a, T b, T c) { return kxor2(a, kxor2(b, c)); }
template <class T>
GL_HD T kandn(T a, T b) { return fo::mul(fo::sub(fo::k<T>(1), a), b); }
template <class T>
GL_HD T kbool(T a) { return fo::mulw(a, fo::sub(a, fo::k<T>(1))); }  // only ever emitted

// Keccak tables for the constraint bodies: rho offsets rot[x*5+y] and the
// round constants, from constant memory (device) or host arrays.
struct KTabDev {
    __device__ static int rot(int i) { return c_keccak_rot[i]; }
    __device__ static uint64_t rc(int r) { return c_keccak_rc[r]; }
};

// Constraint indices (emission order of the AIR's eval; 3182 in total):
//   0..23     first-row flags      24..47  flag rotation     48..147 preimage == a
//   148, 149  export               150..249 preimage continuity
//   250..889  (x,z): bool c, xor c2 (interleaved)
//   890..2589 a limbs: per (y,x,l) 16 bools (z descending) + the limb equation
//   2590..2909 (x,z): sum_y a1 - c2 in {0,2,4}
//   2910..3009 a2 limbs          3010..3077 a2[0][0] bits + limbs
//   3078..3081 a3[0][0] limbs    3082..3181 output == next input (x outer)
// (c2 = C', a1 = A', a2 = A'', a3 = A''' in the Keccak-f round notation.)
constexpr int KEC_TASKS = 1502;  // 832 quarter-limb tasks, 320 (x,z), 350 light

struct KFold {
    gl::Acc c0, c1;  // lazy sums of v * alpha^(K-1-k), reduced once per point
    const uint64_t *ap;
    __device__ __forceinline__ explicit KFold(const uint64_t *a) : ap(a) {}
    __device__ __forceinline__ void emit(int k, uint64_t v) {
        c0.mac(v, __ldg(ap + 2 * k));
        c1.mac(v, __ldg(ap + 2 * k + 1));
    }
};

#pragma nv_exec_check_disable
template <class T, class Tab>
GL_HD T kbit_b(const T *L, int bx, int by, int z) {
    int ax = (bx + 3 * by) % 5;
    int rot = Tab::rot(ax * 5 + bx);
    return L[KC_AP + (bx * 5 + ax) * 64 + ((z + 64 - rot) & 63)];
}

// one task of one point; L, N in shared memory. Limb equations are linear in
// their bits, so a 16-bit limb is split into four 4-bit tasks that each add
// alpha^k * (their part of the limb) to the fold; part 0 also subtracts
// alpha^k * limb. All tasks then cost about the same.
#pragma nv_exec_check_disable
template <class T, class Tab, class F>
GL_HD void keccak_task(int t, const T *L, const T *N, T first, T trans, F &f) {
    const T not_final = fo::sub(fo::k<T>(1), L[KC_STEP + 23]);
    if (t < 400) {  // A limbs from xor(A1, C, C2), with the bools of A1
        int o = t >> 2, part = t & 3, y = o / 20, x = (o / 4) % 5, l = o % 4;
        int base = 890 + 17 * o;
        T acc = fo::k<T>(0);
        for (int z = l * 16 + 4 * part + 3; z >= l * 16 + 4 * part; z--) {
            T ap = L[KC_AP + (y * 5 + x) * 64 + z];
            f.emit(base + (l * 16 + 15 - z), kbool(ap));
            acc = fo::add(fo::dbl(acc), kxor3(ap, L[KC_C + x * 64 + z], L[KC_CP + x * 64 + z]));
        }
        acc = fo::mulc(acc, 1ull << (4 * part));
        f.emit(base + 16, part == 0 ? fo::sub(acc, L[KC_A + o]) : acc);
    } else if (t < 800) {  // A2 limbs: xor(B, andn(B[x+1], B[x+2]))
        int o = (t - 400) >> 2, part = t & 3, y = o / 20, x = (o / 4) % 5, l = o % 4;
        T acc = fo::k<T>(0);
        for (int z = l * 16 + 4 * part + 3; z >= l * 16 + 4 * part; z--) {
            T b0 = kbit_b<T, Tab>(L, x, y, z), b1 = kbit_b<T, Tab>(L, (x + 1) % 5, y, z), b2 = kbit_b<T, Tab>(L, (x + 2) % 5, y, z);
            acc = fo::add(fo::dbl(acc), kxor2(b0, kandn(b1, b2)));
        }
        acc = fo::mulc(acc, 1ull << (4 * part));
        f.emit(2910 + o, part == 0 ? fo::sub(acc, L[KC_APP + o]) : acc);
    } else if (t < 816) {  // A2[0][0] bits
        int l = (t - 800) >> 2, part = t & 3, base = 3010 + 17 * l;
        T acc = fo::k<T>(0);
        for (int z = l * 16 + 4 * part + 3; z >= l * 16 + 4 * part; z--) {
            T bit = L[KC_APP00 + z];
            f.emit(base + (l * 16 + 15 - z), kbool(bit));
            acc = fo::add(fo::dbl(acc), bit);
        }
        acc = fo::mulc(acc, 1ull << (4 * part));
        f.emit(base + 16, part == 0 ? fo::sub(acc, L[KC_APP + l]) : acc);
    } else if (t < 832) {  // A3[0][0] = A2[0][0] xor RC
        int l = (t - 816) >> 2, part = t & 3;
        T acc = fo::k<T>(0);
        for (int z = l * 16 + 4 * part + 3; z >= l * 16 + 4 * part; z--) {
            T rcb = fo::k<T>(0);
            for (int r = 0; r < 24; r++)
                if ((Tab::rc(r) >> z) & 1) rcb = fo::add(rcb, L[KC_STEP + r]);
            acc = fo::add(fo::dbl(acc), kxor2(L[KC_APP00 + z], rcb));
        }
        acc = fo::mulc(acc, 1ull << (4 * part));
        f.emit(3078 + l, part == 0 ? fo::sub(acc, L[KC_APPP00 + l]) : acc);
    } else if (t < 1152) {  // (x, z): bool C, C2 xor, A1 column sum
        int i = t - 832, x = i / 64, z = i % 64;
        T cxz = L[KC_C + i];
        f.emit(250 + 2 * i, kbool(cxz));
        T v = kxor3(cxz, L[KC_C + ((x + 4) % 5) * 64 + z], L[KC_C + ((x + 1) % 5) * 64 + ((z + 63) & 63)]);
        T cp = L[KC_CP + i];
        f.emit(251 + 2 * i, fo::sub(cp, v));
        T sm = fo::k<T>(0);
        for (int y = 0; y < 5; y++) sm = fo::add(sm, L[KC_AP + (y * 5 + x) * 64 + z]);
        T d = fo::sub(sm, cp);
        f.emit(2590 + i, fo::mulw(fo::mul(d, fo::sub(d, fo::k<T>(2))), fo::sub(d, fo::k<T>(4))));
    } else if (t < 1176) {  // first-row flags
        int i = t - 1152;
        f.emit(i, fo::mulw(first, i == 0 ? fo::sub(L[KC_STEP], fo::k<T>(1)) : L[KC_STEP + i]));
    } else if (t < 1200) {  // flag rotation
        int i = t - 1176;
        f.emit(24 + i, fo::mulw(trans, fo::sub(N[KC_STEP + (i + 1) % 24], L[KC_STEP + i])));
    } else if (t < 1300) {  // first step: preimage == a
        int o = t - 1200;
        f.emit(48 + o, fo::mulw(L[KC_STEP], fo::sub(L[KC_PRE + o], L[KC_A + o])));
    } else if (t < 1302) {  // export
        T ex = L[KC_EXPORT];
        if (t == 1300) f.emit(148, kbool(ex));
        else f.emit(149, fo::mulw(not_final, ex));
    } else if (t < 1402) {  // preimage continuity
        int o = t - 1302;
        f.emit(150 + o, fo::mulw(fo::mul(not_final, trans), fo::sub(L[KC_PRE + o], N[KC_PRE + o])));
    } else {  // round output == next round input (x outer, y inner)
        int i = t - 1402, x = i / 20, y = (i / 4) % 5, l = i % 4;
        T outv = (x == 0 && y == 0) ? L[KC_APPP00 + l] : L[KC_APP + (y * 5 + x) * 4 + l];
        f.emit(3082 + i, fo::mulw(fo::mul(not_final, trans), fo::sub(outv, N[KC_A + (y * 5 + x) * 4 + l])));
    }
}

// Persistent blocks over contiguous point ranges. Rows are staged in a ring
// of D + 1 shared-memory slots: point m needs rows m and m + D (D = 2 for
// this AIR alone; up to 8 when it is proved beside an AIR of higher degree),
// so each LDE row is read from HBM once per block range. Selectors for the
// next 256 points are computed cooperatively (one inversion per point).
constexpr int KEC_THREADS = 256;
__global__ void __launch_bounds__(KEC_THREADS) keccak_eval_block_kernel(const __grid_constant__ EvalArgs a,
                                                                         uint64_t points_per_block) {
    extern __shared__ uint64_t sm[];
    const uint32_t slots = (uint32_t)a.D + 1;
    uint64_t *ring = sm;                        // (D + 1) x 2633
    uint64_t *sel = sm + slots * KC_NCOLS;      // 256 x {first, trans}
    uint64_t *red = sel + 2 * KEC_THREADS;      // 8 warps x 2
    const uint64_t qh = 1ull << a.log_qh;
    const uint64_t m0 = (uint64_t)blockIdx.x * points_per_block;
    if (m0 >= qh) return;
    const uint64_t m1 = min(qh, m0 + points_per_block);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    auto load_row = [&](uint64_t m, int slot) {
        const uint64_t *src = a.lde + gl::bitrev(m & (qh - 1), a.log_qh) * a.w;
        uint64_t *dst = ring + slot * KC_NCOLS;
        for (int c = tid; c < KC_NCOLS; c += KEC_THREADS) dst[c] = __ldg(src + c);
    };
    for (uint64_t j = 0; j < a.D; j++) load_row(m0 + j, (int)((m0 + j) % slots));
    for (uint64_t m = m0; m < m1; m++) {
        const uint64_t j = m - m0;
        if ((j & (KEC_THREADS - 1)) == 0) {
            uint64_t pm = m + tid;
            if (pm < m1) {
                uint64_t x = point_x(a, pm);
                sel[2 * tid] = gl::mul(a.zh[pm & (a.D - 1)], gl::inv(gl::sub(x, 1)));
                sel[2 * tid + 1] = gl::sub(x, a.omega_h_inv);
            }
        }
        load_row(m + a.D, (int)((m + a.D) % slots));
        __syncthreads();
        const uint64_t *L = ring + (m % slots) * KC_NCOLS;
        const uint64_t *N = ring + ((m + a.D) % slots) * KC_NCOLS;
        const uint64_t first = sel[2 * (j & (KEC_THREADS - 1))], trans = sel[2 * (j & (KEC_THREADS - 1)) + 1];
        KFold f(a.alpha_pows);
        for (int t = tid; t < KEC_TASKS; t += KEC_THREADS) keccak_task<uint64_t, KTabDev>(t, L, N, first, trans, f);
        uint64_t c0 = f.c0.reduce(), c1 = f.c1.reduce();
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            c0 = gl::add(c0, __shfl_xor_sync(0xffffffffu, c0, off));
            c1 = gl::add(c1, __shfl_xor_sync(0xffffffffu, c1, off));
        }
        if (lane == 0) {
            red[2 * wid] = c0;
            red[2 * wid + 1] = c1;
        }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < KEC_THREADS / 32; w++) {
                c0 = gl::add(c0, red[2 * w]);
                c1 = gl::add(c1, red[2 * w + 1]);
            }
            uint64_t *o = a.acc + 2 * m;
            o[0] = gl::add(o[0], c0);
            o[1] = gl::add(o[1], c1);
        }
        // slot (m % (D + 1)) is overwritten by row m + D + 1 in the next iteration
        __syncthreads();
    }
}
// shared memory of a launch with quotient degree D (at most 8: 194 KB)
inline size_t kec_smem(uint64_t D) { return ((D + 1) * KC_NCOLS + 2 * KEC_THREADS + 16) * 8; }
constexpr size_t KEC_SMEM_MAX = (9 * KC_NCOLS + 2 * KEC_THREADS + 16) * 8;

// acc[0..old) *= beta (EF); then acc[i] = acc[i mod old] for i in [old, new)
__global__ void scale_ef_kernel(uint64_t *acc, uint64_t n, gl::ef beta) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gl::ef v = gl::ef_mul(gl::ef{acc[2 * i], acc[2 * i + 1]}, beta);
    acc[2 * i] = v.c0;
    acc[2 * i + 1] = v.c1;
}
__global__ void tile_ef_kernel(uint64_t *acc, uint64_t old_n, uint64_t new_n) {
    uint64_t i = old_n + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= new_n) return;
    uint64_t s = i & (old_n - 1);
    acc[2 * i] = acc[2 * s];
    acc[2 * i + 1] = acc[2 * s + 1];
}
// numerator[i] *= 1 / Z_H(x_i), Z_H periodic with period D (quotient.rs:380-409)
struct VanArgs {
    uint64_t inv_van[8];
    uint64_t D;
};
__global__ void divide_vanishing_kernel(uint64_t *acc, uint64_t n, const __grid_constant__ VanArgs v) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t s = v.inv_van[i & (v.D - 1)];
    acc[2 * i] = gl::mul(acc[2 * i], s);
    acc[2 * i + 1] = gl::mul(acc[2 * i + 1], s);
}

}  // namespace quot
