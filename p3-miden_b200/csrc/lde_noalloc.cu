// p3g_coset_lde_noalloc: the bit-reversed coset LDE (the same computation as
// p3g_coset_lde) for callers that cannot allocate device memory.
//
// Who needs it: code that runs with a fixed, pre-reserved device-memory
// budget and must not call into the CUDA allocator once it is running — for
// example a proof server that has handed all remaining HBM to its job slots,
// or a host runtime whose own allocator owns the device and forbids
// cudaMalloc/cudaFree (and the implicit synchronisation they bring) on its
// hot path. Such callers pass their input and output buffers; this entry
// point needs nothing else.
//
// Scratch: all intermediate data (the inverse-transform coefficients, the
// twiddle and coset-scaling tables) lives in g_lde_scratch below, a
// file-scope static __device__ array of 16.1 MiB. Every GPU that loads the
// library holds it until the process exits. Limits: height <= 2^22 rows and
// height * width <= 2^21 words; larger calls return P3G_ERR_INVALID before
// any work is queued.
//
// Every call shares the one array, which keeps the last call's contents
// (every word a call reads is first written by that same call). Calls whose
// work overlaps on the GPU — on two streams, or from two threads — race on
// the array and corrupt each other's results; serialise them on one stream.
//
// Set-up: the first call on each device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress and sets the kernels'
// shared-memory limits; make that first call before any stream capture.
// The address is cached for the life of the process: a cudaDeviceReset (or
// any other end of the device's primary context) invalidates it, and this
// entry point does not support calls after one.
// The call is asynchronous on `stream` (0 = the legacy default stream).
//
// Errors: P3G_ERR_INVALID for arguments outside the limits (nothing is
// queued); P3G_ERR_CUDA when a launch fails, or when an error from earlier,
// unrelated work is already pending on this host thread (that error is left
// in place for its owner and nothing is queued).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/p3g.h"
#include "gl.cuh"
#include "ntt.cuh"

namespace {

constexpr uint64_t NOALLOC_MAX_WORDS = 1ull << 21;  // coefficient scratch, height * width
constexpr uint32_t NOALLOC_MAX_LOG_H = 22;
constexpr uint32_t LO_BITS = 12;
constexpr uint64_t LO_LEN = 1ull << LO_BITS;                              // 4096
constexpr uint64_t HI_LEN = 1ull << (NOALLOC_MAX_LOG_H - LO_BITS);        // 1024
// layout of the scratch array (words)
constexpr uint64_t OFF_COEF = 0;
constexpr uint64_t OFF_FWD_LO = OFF_COEF + NOALLOC_MAX_WORDS;
constexpr uint64_t OFF_FWD_HI = OFF_FWD_LO + LO_LEN;
constexpr uint64_t OFF_INV_LO = OFF_FWD_HI + HI_LEN;
constexpr uint64_t OFF_INV_HI = OFF_INV_LO + LO_LEN;
constexpr uint64_t OFF_T1024_FWD = OFF_INV_HI + HI_LEN;
constexpr uint64_t OFF_T1024_INV = OFF_T1024_FWD + 512;
constexpr uint64_t OFF_SCALE_LO = OFF_T1024_INV + 512;
constexpr uint64_t OFF_SCALE_HI = OFF_SCALE_LO + LO_LEN;
constexpr uint64_t NOALLOC_WORDS = OFF_SCALE_HI + HI_LEN;  // 2,113,536 words = 16.1 MiB

static __device__ __align__(256) uint64_t g_lde_scratch[NOALLOC_WORDS];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
uint64_t *g_scratch_ptr[MAX_DEVICES] = {nullptr};

// lo[j] = lo_mul * v^j (j < nlo); hi[j] = v^(nlo * j) (j < nhi)
__global__ void fill_pow_tables_kernel(uint64_t *lo, uint32_t nlo, uint64_t *hi, uint32_t nhi, uint64_t v,
                                       uint64_t lo_mul) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nlo) {
        lo[i] = gl::mul(lo_mul, gl::pow(v, i));
    } else if (i < nlo + nhi) {
        hi[i - nlo] = gl::pow(gl::pow(v, nlo), i - nlo);
    }
}

void fill_tables(uint64_t *lo, uint32_t nlo, uint64_t *hi, uint32_t nhi, uint64_t v, uint64_t lo_mul, cudaStream_t s) {
    uint32_t n = nlo + nhi;
    fill_pow_tables_kernel<<<(n + 255) / 256, 256, 0, s>>>(lo, nlo, hi, nhi, v, lo_mul);
}

template <int C, bool DIF>
void set_smem_limit() {
    cudaFuncSetAttribute(ntt::ntt_pass_kernel<C, DIF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (1024 * C + 512 + 16) * 8);
}

// once per device, with that device current
int setup_device(int dev, uint64_t **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        uint64_t *p = nullptr;
        if (cudaGetSymbolAddress((void **)&p, g_lde_scratch) != cudaSuccess || !p) return P3G_ERR_CUDA;
        set_smem_limit<2, false>();
        set_smem_limit<4, false>();
        set_smem_limit<8, false>();
        set_smem_limit<2, true>();
        set_smem_limit<4, true>();
        set_smem_limit<8, true>();
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return 0;
}

unsigned log2_exact(uint64_t n) {
    unsigned l = 0;
    while ((1ull << l) < n) l++;
    return l;
}

// Column tiles sit on grid.y, whose limit is 65535: a wide matrix is
// launched in column chunks of at most 65535 tiles (the row strides stay the
// full width, so each chunk is the same pass over a column range).
constexpr uint64_t MAX_TILES_Y = 65535;

template <bool DIF>
void launch(const ntt::PassArgs &a, uint64_t h, cudaStream_t s) {
    uint32_t k = a.bhi - a.blo;
    size_t smem_words_per_col = size_t(1) << k;
    if (a.w <= 2) {
        dim3 g((unsigned)(h >> k), (unsigned)((a.w + 1) / 2));
        ntt::ntt_pass_kernel<2, DIF><<<g, 256, (smem_words_per_col * 2 + 512 + 16) * 8, s>>>(a);
    } else if (a.w <= 4) {
        dim3 g((unsigned)(h >> k), (unsigned)((a.w + 3) / 4));
        ntt::ntt_pass_kernel<4, DIF><<<g, 256, (smem_words_per_col * 4 + 512 + 16) * 8, s>>>(a);
    } else {
        for (uint64_t c0 = 0; c0 < a.w; c0 += 8 * MAX_TILES_Y) {
            ntt::PassArgs b = a;
            b.src = a.src + c0;
            b.dst = a.dst + c0;
            b.w = a.w - c0 < 8 * MAX_TILES_Y ? a.w - c0 : 8 * MAX_TILES_Y;
            dim3 g((unsigned)(h >> k), (unsigned)((b.w + 7) / 8));
            ntt::ntt_pass_kernel<8, DIF><<<g, 256, (smem_words_per_col * 8 + 512 + 16) * 8, s>>>(b);
        }
    }
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int p3g_coset_lde_noalloc(const uint64_t *d_in, uint64_t height,
                                                                         uint64_t width, uint32_t log_blowup,
                                                                         uint64_t shift, uint64_t *d_out,
                                                                         void *stream) {
    if (!d_in || !d_out || height == 0 || (height & (height - 1)) || width == 0) return P3G_ERR_INVALID;
    const uint32_t L = log2_exact(height);
    if (L > NOALLOC_MAX_LOG_H || log_blowup > 8 || L + log_blowup > 32) return P3G_ERR_INVALID;
    if (width > NOALLOC_MAX_WORDS || height * width > NOALLOC_MAX_WORDS) return P3G_ERR_INVALID;
    // an error left by earlier work on this thread is not this call's: report
    // it without clearing it, and queue nothing
    if (cudaPeekAtLastError() != cudaSuccess) return P3G_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return P3G_ERR_CUDA;
    uint64_t *S = nullptr;
    if (setup_device(dev, &S)) return P3G_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    shift %= gl::P;

    const uint32_t lo_bits = L < LO_BITS ? L : LO_BITS;
    const uint32_t nlo = 1u << lo_bits, nhi = 1u << (L - lo_bits);
    const uint64_t w_root = gl::root(L);
    fill_tables(S + OFF_FWD_LO, nlo, S + OFF_FWD_HI, nhi, w_root, 1, s);
    fill_tables(S + OFF_INV_LO, nlo, S + OFF_INV_HI, nhi, gl::inv(w_root), 1, s);
    fill_tables(S + OFF_T1024_FWD, 512, nullptr, 0, gl::root(10), 1, s);
    fill_tables(S + OFF_T1024_INV, 512, nullptr, 0, gl::inv(gl::root(10)), 1, s);

    // passes of at most 10 bits, sizes as even as possible
    uint32_t np = L == 0 ? 1 : (L + 9) / 10, sizes[4];
    for (uint32_t i = 0; i < np; i++) sizes[i] = L / np + (i < L % np ? 1 : 0);

    uint64_t *coef = S + OFF_COEF;
    // inverse transform (DIT): input rows read bit-reversed, natural-order coefficients
    uint32_t blo = 0;
    for (uint32_t pi = 0; pi < np; pi++) {
        ntt::PassArgs a{};
        a.src = pi == 0 ? d_in : coef;
        a.ld_src = width;
        a.dst = coef;
        a.ld_dst = width;
        a.w = width;
        a.L = L;
        a.blo = blo;
        a.bhi = blo + sizes[pi];
        a.src_bitrev = pi == 0;
        a.tw = ntt::PowTab{S + OFF_INV_LO, S + OFF_INV_HI, lo_bits};
        a.tw1024 = S + OFF_T1024_INV;
        a.has_scale = 0;
        launch<false>(a, height, s);
        blo = a.bhi;
    }
    // forward transform per coset (DIF) straight into the caller's output
    const uint64_t wb = gl::root(L + log_blowup);
    const uint64_t hinv = gl::inv(height % gl::P);
    uint64_t sk = shift;
    for (uint64_t k = 0; k < (1ull << log_blowup); k++) {
        fill_tables(S + OFF_SCALE_LO, nlo, S + OFF_SCALE_HI, nhi, sk, hinv, s);
        uint64_t *blk = d_out + gl::bitrev(k, log_blowup) * height * width;
        uint32_t bhi = L;
        for (uint32_t pi = 0; pi < np; pi++) {
            ntt::PassArgs a{};
            a.src = pi == 0 ? coef : blk;
            a.ld_src = width;
            a.dst = blk;
            a.ld_dst = width;
            a.w = width;
            a.L = L;
            a.bhi = bhi;
            a.blo = bhi - sizes[pi];
            a.src_bitrev = 0;
            a.tw = ntt::PowTab{S + OFF_FWD_LO, S + OFF_FWD_HI, lo_bits};
            a.tw1024 = S + OFF_T1024_FWD;
            a.has_scale = pi == 0;
            a.scale = ntt::PowTab{S + OFF_SCALE_LO, S + OFF_SCALE_HI, lo_bits};
            launch<true>(a, height, s);
            bhi = a.blo;
        }
        sk = gl::mul(sk, wb);
    }
    return cudaGetLastError() == cudaSuccess ? P3G_OK : P3G_ERR_CUDA;
}

extern "C" __attribute__((visibility("default"))) uint64_t p3g_coset_lde_noalloc_max_words(void) {
    return NOALLOC_MAX_WORDS;
}
