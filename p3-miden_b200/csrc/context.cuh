// Device context: stream, stream-ordered allocations, twiddle tables, and
// the host drivers for the LDE and LMCS tree kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <chrono>
#include <map>
#include <mutex>
#include <memory>
#include <string>
#include <vector>

#include "gl.cuh"
#include "merkle.cuh"
#include "lde.cuh"
#include "ntt.cuh"
#include "poseidon2.cuh"

namespace p3g {

enum Status : int {
    OK = 0,
    ERR_INVALID = 1,     // bad argument (null pointer, size, unsupported parameter)
    ERR_VALIDATION = 2,  // instance validation failed (AIR, height order, width)
    ERR_OOM = 3,         // device allocation refused
    ERR_TIMEOUT = 4,     // a bounded device-side search gave up
    ERR_CUDA = 5,        // other CUDA runtime error
    ERR_REJECTED = 6,    // the server's self-check rejected the proof
};

struct CudaError {
    int status;
    std::string what;
};

inline void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        int st = (e == cudaErrorMemoryAllocation) ? ERR_OOM : ERR_CUDA;
        throw CudaError{st, std::string(what) + ": " + cudaGetErrorString(e)};
    }
}
#define CK(x) ::p3g::check((x), #x)

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) for a kernel, once per
// device (function attributes belong to each device's copy of the module);
// `done` is the call site's bit set of devices already set.
template <typename K>
inline void smem_attr_once(std::atomic<uint64_t> &done, K kernel, int bytes) {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "cudaFuncSetAttribute");
    done.fetch_or(bit, std::memory_order_release);
}

inline unsigned log2u(uint64_t n) {
    unsigned l = 0;
    while ((1ull << l) < n) l++;
    return l;
}

// Buffer cache of a context. Repeated proofs of one shape allocate the same
// large buffers every time; from the pool, such allocations now and then
// stalled the host for 10-100 ms (the pool's reserved memory did not grow).
// Buffers of at least kMinWords allocated and released on the context's own
// stream are kept, up to limit_words, and handed out again for an allocation
// of exactly the same size on that stream: stream order makes that reuse as
// safe as the pool's own same-stream reuse. Buffers released after the
// context is gone (alive false) are freed as before.
struct BufCache {
    static constexpr size_t kMinWords = 1ull << 20;  // 8 MB
    bool alive = true;
    cudaStream_t home = nullptr;
    size_t limit_words = 0, cached_words = 0;
    std::multimap<size_t, uint64_t *> free;
    bool put(uint64_t *p, size_t words, cudaStream_t s) {
        if (!alive || s != home || words < kMinWords || cached_words + words > limit_words) return false;
        free.insert({words, p});
        cached_words += words;
        return true;
    }
    uint64_t *take(size_t words) {
        auto it = free.find(words);
        if (it == free.end()) return nullptr;
        uint64_t *p = it->second;
        free.erase(it);
        cached_words -= words;
        return p;
    }
    void clear() {
        for (auto &e : free) cudaFreeAsync(e.second, home);
        free.clear();
        cached_words = 0;
    }
};

// A device buffer owned by a context, freed stream-ordered.
struct DBuf {
    uint64_t *p = nullptr;
    size_t words = 0;
    cudaStream_t s = nullptr;
    std::shared_ptr<BufCache> cache;  // where the buffer goes back to, or null
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : p(o.p), words(o.words), s(o.s), cache(std::move(o.cache)) { o.p = nullptr; }
    DBuf &operator=(DBuf &&o) noexcept {
        release();
        p = o.p, words = o.words, s = o.s, cache = std::move(o.cache);
        o.p = nullptr;
        return *this;
    }
    void release() {
        if (p && !(cache && cache->put(p, words, s))) cudaFreeAsync(p, s);
        p = nullptr;
        cache.reset();
    }
    ~DBuf() { release(); }
};

struct TwTables {
    DBuf fwd_lo, fwd_hi, inv_lo, inv_hi;
    uint32_t lo_bits;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t p2[p2::N_PARAMS];
    std::map<uint32_t, std::unique_ptr<TwTables>> tw;
    std::string last_error;
    uint64_t *pinned = nullptr;  // small pinned staging area
    size_t pinned_words = 0;
    uint64_t launches = 0;       // kernels launched by this context
    cudaStream_t lde_stream = nullptr, copy_stream = nullptr;  // main-commit pipeline
    // Tuned launch shapes (p3g_autotune / p3g_ctx_set_*): the bit ranges of
    // an LDE of 2^L rows, and the column-slab width of the main commit (0:
    // the default of about 8 slabs for wide traces). Results do not depend on
    // them: every choice computes the same values.
    std::map<uint32_t, std::vector<uint32_t>> lde_split;
    uint64_t slab_cols = 0;
    // DAG nodes per generated constraint kernel of the symbolic AIRs created
    // on this context (0: the default, 500)
    uint64_t air_chunk_nodes = 0;

    // This context's own stream-ordered memory pool. Buffers freed by one
    // context are reused only by that context, so two contexts driving the
    // same device (server workers) never wait on each other's frees, and the
    // memory goes back to the device when the context is released. Freed
    // blocks stay in the pool between proofs (release threshold: unlimited).
    cudaMemPool_t pool = nullptr;
    void make_pool() {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        CK(cudaMemPoolCreate(&pool, &props));
        uint64_t thr = UINT64_MAX;
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    }
    void pipeline_streams() {
        if (!lde_stream) CK(cudaStreamCreateWithFlags(&lde_stream, cudaStreamNonBlocking));
        if (!copy_stream) CK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    }
    // Buffer cache (BufCache) on the context's own stream; off until
    // enable_cache is called.
    std::shared_ptr<BufCache> bc;
    void enable_cache(size_t limit_words) {
        bc = std::make_shared<BufCache>();
        bc->home = stream;
        bc->limit_words = limit_words;
    }

    // free stream-ordered buffers, then the streams (used at teardown)
    void release() {
        if (stream) cudaStreamSynchronize(stream);
        if (lde_stream) cudaStreamSynchronize(lde_stream);
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        tw.clear();
        ws.release();
        if (bc) {
            bc->clear();
            bc->alive = false;
            bc.reset();
        }
        if (stream) cudaStreamSynchronize(stream);
        if (pinned) cudaFreeHost(pinned);
        pinned = nullptr;
        if (lde_stream) cudaStreamDestroy(lde_stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (stream) cudaStreamDestroy(stream);
        lde_stream = copy_stream = stream = nullptr;
        // buffers still held elsewhere (a tree the caller has not freed) keep
        // the pool alive until they are freed
        if (pool) cudaMemPoolDestroy(pool);
        pool = nullptr;
    }

    // Workspace kept between proofs: the column-major copies of the LDE rows
    // that the generated constraint kernels read. Allocating and freeing a
    // multi-GB buffer every proof made the pool's allocation calls stall the
    // host for up to about 0.1 s now and then; kept, it is allocated once.
    DBuf ws;
    uint64_t *workspace(size_t words) {
        if (ws.words < words) {
            ws.release();
            ws = alloc(words);
        }
        return ws.p;
    }
    double alloc_ms = 0;  // host time spent in device allocation calls (memory statistics)
    DBuf alloc(size_t words) {
        DBuf b;
        b.s = stream;
        b.words = words;
        if (bc && stream == bc->home) {
            b.cache = bc;
            if (words >= BufCache::kMinWords && (b.p = bc->take(words))) return b;
        }
        if (words) {
            const auto t0 = std::chrono::steady_clock::now();
            if (pool) CK(cudaMallocFromPoolAsync((void **)&b.p, words * 8, pool, stream));
            else CK(cudaMallocAsync((void **)&b.p, words * 8, stream));
            alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        return b;
    }
    uint64_t *stage(size_t words) {
        if (words > pinned_words) {
            if (pinned) {
                CK(cudaStreamSynchronize(stream));
                cudaFreeHost(pinned);
            }
            pinned_words = words < 4096 ? 4096 : words;
            CK(cudaMallocHost((void **)&pinned, pinned_words * 8));
        }
        return pinned;
    }
    void h2d(uint64_t *dst, const uint64_t *src, size_t words) {
        if (words) CK(cudaMemcpyAsync(dst, src, words * 8, cudaMemcpyHostToDevice, stream));
    }
    void d2h(uint64_t *dst, const uint64_t *src, size_t words) {
        if (words) CK(cudaMemcpyAsync(dst, src, words * 8, cudaMemcpyDeviceToHost, stream));
    }
    void sync() { CK(cudaStreamSynchronize(stream)); }
    // upload a small host vector to a fresh device buffer
    DBuf upload(const std::vector<uint64_t> &v) {
        DBuf b = alloc(v.size());
        uint64_t *st = stage(v.size());
        CK(cudaStreamSynchronize(stream));
        memcpy(st, v.data(), v.size() * 8);
        h2d(b.p, st, v.size());
        CK(cudaStreamSynchronize(stream));
        return b;
    }

    // Two-level tables of powers of w_{2^L} and its inverse.
    const TwTables &twiddles(uint32_t L) {
        auto it = tw.find(L);
        if (it != tw.end()) return *it->second;
        auto t = std::make_unique<TwTables>();
        uint32_t lo_bits = L < 12 ? L : 12;
        t->lo_bits = lo_bits;
        uint64_t w = gl::root(L), wi = gl::inv(w);
        size_t nlo = 1ull << lo_bits, nhi = 1ull << (L - lo_bits);
        std::vector<uint64_t> a(nlo), b(nhi), c(nlo), d(nhi);
        uint64_t x = 1, y = 1;
        for (size_t i = 0; i < nlo; i++) a[i] = x, c[i] = y, x = gl::mul(x, w), y = gl::mul(y, wi);
        uint64_t W = x, WI = y;  // w^(2^lo_bits)
        x = 1, y = 1;
        for (size_t i = 0; i < nhi; i++) b[i] = x, d[i] = y, x = gl::mul(x, W), y = gl::mul(y, WI);
        t->fwd_lo = upload(a);
        t->fwd_hi = upload(b);
        t->inv_lo = upload(c);
        t->inv_hi = upload(d);
        auto &ref = *t;
        tw[L] = std::move(t);
        return ref;
    }
};

// The permutation constants live in the __constant__ table c_p2, one copy
// per device for the whole process. Each context keeps its own constants
// (the StarkConfig's permutation) and makes them current on its device
// before launching kernels that hash; the upload happens only when a context
// with different constants ran last on that device. Contexts whose constants
// differ must therefore not have hashing kernels in flight at the same time.
inline void bind_p2(const Ctx &ctx) {
    static std::mutex mu;
    static std::map<int, std::vector<uint64_t>> bound;
    std::lock_guard<std::mutex> lk(mu);
    std::vector<uint64_t> &b = bound[ctx.device];
    if (b.size() == p2::N_PARAMS && memcmp(b.data(), ctx.p2, sizeof(ctx.p2)) == 0) return;
    CK(cudaSetDevice(ctx.device));
    CK(cudaDeviceSynchronize());  // kernels of the previous constants finish first
    CK(cudaMemcpyToSymbol(c_p2, ctx.p2, sizeof(ctx.p2)));
    b.assign(ctx.p2, ctx.p2 + p2::N_PARAMS);
}

// out[r] = in[bitrev(r)] for the rows of an n x w matrix (n = 2^L)
__global__ void bitrev_rows_kernel(const uint64_t *in, uint64_t *out, uint32_t L, uint64_t w) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >> L >= w) return;
    const uint64_t r = i / w, c = i % w;
    out[r * w + c] = in[gl::bitrev(r, L) * w + c];
}

// Column-major copy of the first n rows of a row-major matrix of w columns
// (row stride ld words): out[c * n + r] = in[r * ld + c]. 32 x 32 tiles
// through shared memory, rows on grid.x and column tiles on grid.y; both the
// loads (32 columns of a row) and the stores (32 rows of a column) are
// 256-byte runs.
__global__ void __launch_bounds__(256) transpose_kernel(const uint64_t *in, uint64_t ld, uint64_t *out, uint64_t n,
                                                        uint64_t w) {
    __shared__ uint64_t t[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.x * 32, c0 = (uint64_t)blockIdx.y * 32;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (uint32_t j = 0; j < 32; j += 8) {
        const uint64_t r = r0 + ty + j, c = c0 + tx;
        if (r < n && c < w) t[ty + j][tx] = __ldg(in + r * ld + c);
    }
    __syncthreads();
#pragma unroll
    for (uint32_t j = 0; j < 32; j += 8) {
        const uint64_t c = c0 + ty + j, r = r0 + tx;
        if (r < n && c < w) out[c * n + r] = t[tx][ty + j];
    }
}
inline void transpose(Ctx &ctx, const uint64_t *in, uint64_t ld, uint64_t *out, uint64_t n, uint64_t w) {
    if (!n || !w) return;
    if ((w + 31) / 32 > 65535) throw CudaError{ERR_INVALID, "transpose: too many columns"};
    transpose_kernel<<<dim3((unsigned)((n + 31) / 32), (unsigned)((w + 31) / 32)), dim3(32, 8), 0, ctx.stream>>>(
        in, ld, out, n, w);
    CK(cudaGetLastError());
    ctx.launches++;
}

// Host-built two-level power table of v for exponents < 2^L.
inline void pow_table(uint64_t v, uint32_t L, uint32_t lo_bits, std::vector<uint64_t> &out_lo,
                      std::vector<uint64_t> &out_hi) {
    size_t nlo = 1ull << lo_bits, nhi = 1ull << (L > lo_bits ? L - lo_bits : 0);
    out_lo.resize(nlo);
    out_hi.resize(nhi);
    uint64_t x = 1;
    for (size_t i = 0; i < nlo; i++) out_lo[i] = x, x = gl::mul(x, v);
    uint64_t y = 1;
    for (size_t i = 0; i < nhi; i++) out_hi[i] = y, y = gl::mul(y, x);
}

// A split of L bits into LDE bit ranges is valid when every range has 1..10
// bits (the kernels' shared-memory groups) and the ranges add up to L.
inline bool valid_split(uint32_t L, const std::vector<uint32_t> &sizes) {
    if (sizes.empty() || sizes.size() > 8) return false;
    uint32_t sum = 0;
    for (uint32_t k : sizes) {
        if (k == 0 || k > 10) return false;
        sum += k;
    }
    return sum == L;
}

// split L bits into n ranges, sizes as even as possible
inline std::vector<uint32_t> pass_sizes_n(uint32_t L, uint32_t n) {
    std::vector<uint32_t> v(n, L / n);
    for (uint32_t i = 0; i < L % n; i++) v[i]++;
    return v;
}
// split L bits into passes of at most 10 bits, sizes as even as possible
inline std::vector<uint32_t> pass_sizes(uint32_t L) {
    uint32_t n = L == 0 ? 1 : (L + 9) / 10;
    std::vector<uint32_t> v(n, L / n);
    for (uint32_t i = 0; i < L % n; i++) v[i]++;
    return v;
}

// Bit-reversed coset LDE of an h x w matrix, split into a plan (tables on
// the device; synchronises the context stream once) and launches (no host
// synchronisation, any stream), so that column slabs of one trace can be
// transformed while earlier slabs are hashed.
struct LdePlan {
    uint32_t L = 0, log_blowup = 0;
    uint64_t h = 0;
    std::vector<uint32_t> sizes;  // bit ranges, ascending
    const TwTables *tw = nullptr;
    uint32_t scale_lo_bits = 0;
    uint64_t scale_hi_len = 0;
    DBuf scale_lo, scale_hi;  // every coset's two-level table of (s*w_{hB}^c)^i / h
    DBuf colpow_lo, colpow_hi;
    uint32_t colpow_lo_bits = 0;
    uint64_t colpow_hi_len = 0;
};

// col_bases: if non-empty, coefficient k of base column col is also
// multiplied by col_bases[col/2]^k (quotient chunks).
inline LdePlan lde_plan(Ctx &ctx, uint64_t h, uint32_t log_blowup, uint64_t shift,
                        const std::vector<uint64_t> &col_bases = {}) {
    LdePlan p;
    p.L = log2u(h);
    p.h = h;
    p.log_blowup = log_blowup;
    p.tw = &ctx.twiddles(p.L);
    auto tuned = ctx.lde_split.find(p.L);
    p.sizes = tuned != ctx.lde_split.end() ? tuned->second : pass_sizes(p.L);
    p.scale_lo_bits = p.L < 12 ? p.L : 12;
    const uint64_t wb = gl::root(p.L + log_blowup);
    const uint64_t hinv = gl::inv(h % gl::P);
    std::vector<uint64_t> lo, hi, all_lo, all_hi;
    uint64_t sk = shift;
    for (uint64_t k = 0; k < (1ull << log_blowup); k++) {
        pow_table(sk, p.L, p.scale_lo_bits, lo, hi);
        for (auto &v : lo) v = gl::mul(v, hinv);  // the inverse transform's 1/h
        all_lo.insert(all_lo.end(), lo.begin(), lo.end());
        all_hi.insert(all_hi.end(), hi.begin(), hi.end());
        p.scale_hi_len = hi.size();
        sk = gl::mul(sk, wb);
    }
    p.scale_lo = ctx.upload(all_lo);
    p.scale_hi = ctx.upload(all_hi);
    if (!col_bases.empty()) {
        p.colpow_lo_bits = p.L < 10 ? p.L : 10;
        p.colpow_hi_len = 1ull << (p.L - p.colpow_lo_bits);
        all_lo.clear(), all_hi.clear();
        for (uint64_t cb : col_bases) {
            pow_table(cb, p.L, p.colpow_lo_bits, lo, hi);
            all_lo.insert(all_lo.end(), lo.begin(), lo.end());
            all_hi.insert(all_hi.end(), hi.begin(), hi.end());
        }
        p.colpow_lo = ctx.upload(all_lo);
        p.colpow_hi = ctx.upload(all_hi);
    }
    return p;
}

// KT: the range's bit count as a template argument (0 = read at run time);
// the common 8-column ranges of 7..10 bits get their own instances, whose
// round loops and index arithmetic fold at compile time.
template <int C, bool DIF, int KT = 0>
inline void launch_lde_pass(Ctx &ctx, const lde::PassArgs &a, uint64_t groups, unsigned n_blocks_y) {
    const uint32_t G = 1u << a.k;
    const unsigned threads = (G >= 8 ? G / 8 : 1) * C;
    const size_t smem = ((size_t)G * C + G) * 8;
    static std::atomic<uint64_t> attr_done{0};
    smem_attr_once(attr_done, lde::lde_pass_kernel<C, DIF, KT>, (1024 * C + 1024) * 8);
    lde::lde_pass_kernel<C, DIF, KT><<<dim3((unsigned)(groups * a.n_tiles), n_blocks_y), threads, smem, ctx.stream>>>(a);
    CK(cudaGetLastError());
    ctx.launches++;
}
template <int C, int KT = 0>
inline void launch_lde_fused(Ctx &ctx, const lde::FusedArgs &a, uint64_t groups) {
    const uint32_t G = 1u << a.k;
    const unsigned threads = (G >= 8 ? G / 8 : 1) * C;
    const size_t smem = (2 * (size_t)G * C + 3 * (size_t)G) * 8;
    static std::atomic<uint64_t> attr_done{0};
    smem_attr_once(attr_done, lde::lde_fused_kernel<C, KT>, (2 * 1024 * C + 3 * 1024) * 8);
    lde::lde_fused_kernel<C, KT><<<(unsigned)(groups * a.n_tiles), threads, smem, ctx.stream>>>(a);
    CK(cudaGetLastError());
    ctx.launches++;
}
template <bool DIF>
inline void launch_lde_pass_any(Ctx &ctx, uint32_t C, const lde::PassArgs &a, uint64_t groups, unsigned ny) {
    if (C == 2) launch_lde_pass<2, DIF>(ctx, a, groups, ny);
    else if (C == 4) launch_lde_pass<4, DIF>(ctx, a, groups, ny);
    else if (a.k == 7) launch_lde_pass<8, DIF, 7>(ctx, a, groups, ny);
    else if (a.k == 8) launch_lde_pass<8, DIF, 8>(ctx, a, groups, ny);
    else if (a.k == 9) launch_lde_pass<8, DIF, 9>(ctx, a, groups, ny);
    else if (a.k == 10) launch_lde_pass<8, DIF, 10>(ctx, a, groups, ny);
    else launch_lde_pass<8, DIF>(ctx, a, groups, ny);
}

// in: h x w (row stride ld_in) -> out: (h << log_blowup) x w (row stride
// ld_out); tmp holds h * w words (used when h > 2^10).
inline void lde_run(Ctx &ctx, const LdePlan &p, const uint64_t *d_in, uint64_t ld_in, uint64_t w, uint64_t *d_out,
                    uint64_t ld_out, uint64_t *d_tmp, cudaStream_t stream) {
    if (w == 0) return;
    cudaStream_t saved = ctx.stream;
    ctx.stream = stream;  // launch helpers use ctx.stream
    const uint32_t L = p.L, n = (uint32_t)p.sizes.size();
    const uint64_t h = p.h;
    const uint32_t C = w <= 2 ? 2 : w <= 4 ? 4 : 8;
    const uint32_t n_tiles = (uint32_t)((w + C - 1) / C);
    const ntt::PowTab inv{p.tw->inv_lo.p, p.tw->inv_hi.p, p.tw->lo_bits};
    const ntt::PowTab fwd{p.tw->fwd_lo.p, p.tw->fwd_hi.p, p.tw->lo_bits};
    std::vector<uint32_t> blo(n, 0);
    for (uint32_t i = 1; i < n; i++) blo[i] = blo[i - 1] + p.sizes[i - 1];
    for (uint32_t i = 0; i + 1 < n; i++) {  // inverse transform, low ranges
        lde::PassArgs a{};
        a.src = i == 0 ? d_in : d_tmp;
        a.ld_src = i == 0 ? ld_in : w;
        a.dst = d_tmp;
        a.ld_dst = w;
        a.w = w;
        a.L = L;
        a.blo = blo[i];
        a.k = p.sizes[i];
        a.n_tiles = n_tiles;
        a.src_bitrev = i == 0;
        a.root = inv;
        launch_lde_pass_any<false>(ctx, C, a, h >> a.k, 1);
    }
    {  // top range: inverse, then every coset's scale and forward range
        lde::FusedArgs f{};
        f.src = n == 1 ? d_in : d_tmp;
        f.ld_src = n == 1 ? ld_in : w;
        f.src_bitrev = n == 1;
        f.dst = d_out;
        f.ld_dst = ld_out;
        f.w = w;
        f.L = L;
        f.blo = blo[n - 1];
        f.k = p.sizes[n - 1];
        f.n_tiles = n_tiles;
        f.log_cosets = p.log_blowup;
        f.inv_root = inv;
        f.fwd_root = fwd;
        f.scale_lo = p.scale_lo.p;
        f.scale_hi = p.scale_hi.p;
        f.scale_lo_bits = p.scale_lo_bits;
        f.scale_hi_len = p.scale_hi_len;
        f.cp_lo = p.colpow_lo.p;
        f.cp_hi = p.colpow_hi.p;
        f.cp_lo_bits = p.colpow_lo_bits;
        f.cp_hi_len = p.colpow_hi_len;
        if (C == 2) launch_lde_fused<2>(ctx, f, h >> f.k);
        else if (C == 4) launch_lde_fused<4>(ctx, f, h >> f.k);
        else if (f.k == 7) launch_lde_fused<8, 7>(ctx, f, h >> f.k);
        else if (f.k == 8) launch_lde_fused<8, 8>(ctx, f, h >> f.k);
        else if (f.k == 9) launch_lde_fused<8, 9>(ctx, f, h >> f.k);
        else if (f.k == 10) launch_lde_fused<8, 10>(ctx, f, h >> f.k);
        else launch_lde_fused<8>(ctx, f, h >> f.k);
    }
    for (int i = (int)n - 2; i >= 0; i--) {  // forward transform, low ranges, every coset
        lde::PassArgs a{};
        a.src = d_out;
        a.dst = d_out;
        a.ld_src = a.ld_dst = ld_out;
        a.src_blk = a.dst_blk = h * ld_out;
        a.w = w;
        a.L = L;
        a.blo = blo[i];
        a.k = p.sizes[i];
        a.n_tiles = n_tiles;
        a.src_bitrev = 0;
        a.root = fwd;
        launch_lde_pass_any<true>(ctx, C, a, h >> a.k, 1u << p.log_blowup);
    }
    ctx.stream = saved;
}

// One-shot form on the context stream.
inline void coset_lde(Ctx &ctx, const uint64_t *d_in, uint64_t ld_in, uint64_t h, uint64_t w, uint32_t log_blowup,
                      uint64_t shift, uint64_t *d_out, uint64_t *d_tmp, const std::vector<uint64_t> &col_bases = {}) {
    if (w == 0) return;
    LdePlan p = lde_plan(ctx, h, log_blowup, shift, col_bases);
    lde_run(ctx, p, d_in, ld_in, w, d_out, w, d_tmp, ctx.stream);
}

// ------------------------------------------------------------------ trees
struct Mat {
    const uint64_t *d;  // device, row-major, stride = width
    uint64_t h, w;
};
struct Tree {
    DBuf layers;
    uint32_t depth = 0;
    uint64_t H = 0;
    uint32_t alignment = 1;
    std::vector<Mat> mats;
    Mat salt{nullptr, 0, 0};  // hiding LMCS: H x SALT per-leaf salt, absorbed last (borrowed)
    uint64_t root[4] = {0, 0, 0, 0};
    uint64_t layer_off(uint32_t l) const { return 2 * H - 2 * (H >> l); }
};

// Leaf sponge of one height class of n leaves: one thread per leaf, or one
// 16-lane group per leaf when the class is small (latency-bound).
inline void launch_leaf_class(Ctx &ctx, const merkle::ClassArgs &a, uint64_t n) {
    const unsigned coop_blocks = (unsigned)((n * 16 + 127) / 128), blocks = (unsigned)((n + 127) / 128);
    if (a.cm && a.n_mats != 1) throw CudaError{ERR_INVALID, "column-major copy of a multi-matrix class"};
    if (n <= merkle::kCoopLeaves) {
        if (a.cm) merkle::leaf_class_coop_kernel<true><<<coop_blocks, 128, 0, ctx.stream>>>(a);
        else merkle::leaf_class_coop_kernel<false><<<coop_blocks, 128, 0, ctx.stream>>>(a);
    } else {
        if (a.cm) merkle::leaf_class_kernel<true><<<blocks, 128, 0, ctx.stream>>>(a);
        else merkle::leaf_class_kernel<false><<<blocks, 128, 0, ctx.stream>>>(a);
    }
    CK(cudaGetLastError());
    ctx.launches++;
}

// Compress layer 0 (already filled) up to the root (kernels only; the root
// stays on the device); finish_tree also fetches the root. Levels with at
// least kWideParents parents run one thread per parent, up to four levels
// per launch (a block keeps at least a warp's worth of parents per level);
// levels above 128 parents run one 16-lane group per parent, one launch per
// level; the last levels (at most 128 parents) run in one cluster launch.
constexpr uint64_t kWideParents = 8192;
inline void compress_layers(Ctx &ctx, Tree &t) {
    uint32_t l = 0;
    while (l < t.depth && (t.H >> (l + 1)) >= kWideParents) {
        const uint64_t n_parents = t.H >> (l + 1);
        const uint32_t blk = 256;
        const uint32_t levels = std::min<uint32_t>({4u, log2u(n_parents) - log2u(kWideParents) + 1, t.depth - l});
        merkle::compress_kernel<<<(unsigned)(n_parents / blk), blk, 0, ctx.stream>>>(t.layers.p, t.H, l, levels);
        CK(cudaGetLastError());
        ctx.launches++;
        l += levels;
    }
    while (l < t.depth && (t.H >> (l + 1)) > 128) {
        const uint64_t n_parents = t.H >> (l + 1);
        merkle::compress_level_coop_kernel<<<(unsigned)((n_parents * 16 + 127) / 128), 128, 0, ctx.stream>>>(
            t.layers.p, t.H, l);
        CK(cudaGetLastError());
        ctx.launches++;
        l++;
    }
    if (l < t.depth) {
        merkle::compress_top_kernel<<<merkle::kTopCtas, merkle::kTopThreads, 0, ctx.stream>>>(t.layers.p, t.H, l,
                                                                                             t.depth);
        CK(cudaGetLastError());
        ctx.launches++;
    }
}
inline void finish_tree(Ctx &ctx, Tree &t) {
    compress_layers(ctx, t);
    ctx.d2h(ctx.stage(4), t.layers.p + 4 * t.layer_off(t.depth), 4);
    ctx.sync();
    memcpy(t.root, ctx.pinned, 32);
}

// LMCS tree of matrices that are identically zero (the dummy aux traces).
// Every leaf absorbs the same zero rows (one zero-padded 8-word chunk per 8
// columns of each matrix, overwrite mode), so layer 0 is one digest c_0
// repeated and layer l + 1 is c_{l+1} = compress(c_l, c_l). The depth + 1
// digests are computed on the host and written into the usual layer buffer,
// so openings read it like any other tree; the result equals build_tree's.
inline void build_zero_tree(Ctx &ctx, Tree &t, const std::vector<Mat> &mats, uint32_t alignment) {
    t.mats = mats;
    t.alignment = alignment ? alignment : 1;
    t.H = mats.back().h;
    t.depth = log2u(t.H);
    t.layers = ctx.alloc((2 * t.H - 1) * 4);
    uint64_t s[12] = {0};
    for (const Mat &m : mats)
        for (uint64_t i = 0; i < m.w; i += 8) {
            for (int j = 0; j < 8; j++) s[j] = 0;
            p2::host::permute(s, ctx.p2);
        }
    std::vector<uint64_t> c(4 * (t.depth + 1));
    for (int j = 0; j < 4; j++) c[j] = s[j];
    for (uint32_t l = 0; l < t.depth; l++) {
        uint64_t u[12] = {0};
        for (int j = 0; j < 4; j++) u[j] = u[4 + j] = c[4 * l + j];
        p2::host::permute(u, ctx.p2);
        for (int j = 0; j < 4; j++) c[4 * (l + 1) + j] = u[j];
    }
    DBuf dc = ctx.upload(c);
    const uint64_t n = 2 * t.H - 1;
    merkle::fill_const_layers_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx.stream>>>(t.layers.p, t.H, t.depth, dc.p);
    CK(cudaGetLastError());
    ctx.launches++;
    memcpy(t.root, &c[4 * t.depth], 32);
}

// With `salt` (hiding LMCS, p3-miden-lmcs/src/hiding_lmcs.rs:59-189 and
// lifted_tree.rs:265-283): after every matrix, each leaf absorbs its salt row
// (one more overwrite-mode absorb call), then squeezes.
inline void build_tree(Ctx &ctx, Tree &t, const std::vector<Mat> &mats_in, uint32_t alignment,
                       const Mat *salt = nullptr) {
    t.mats = mats_in;
    t.alignment = alignment ? alignment : 1;
    t.H = mats_in.back().h;
    t.depth = log2u(t.H);
    t.layers = ctx.alloc((2 * t.H - 1) * 4);
    std::vector<Mat> mats = mats_in;  // absorption order: the matrices, then the salt
    if (salt) {
        t.salt = *salt;
        mats.push_back(*salt);
    }
    // height classes in order; at most MAX_MATS matrices per launch
    struct Launch {
        std::vector<size_t> idx;
        uint64_t h;
    };
    std::vector<Launch> launches;
    for (size_t i = 0; i < mats.size(); i++) {
        if (launches.empty() || launches.back().h != mats[i].h || launches.back().idx.size() == merkle::MAX_MATS)
            launches.push_back({{}, mats[i].h});
        launches.back().idx.push_back(i);
    }
    uint64_t max_state_h = 0;
    for (size_t li = 0; li + 1 < launches.size(); li++) max_state_h = std::max(max_state_h, launches[li].h);
    DBuf st_a, st_b;
    if (max_state_h) {
        st_a = ctx.alloc(max_state_h * 12);
        st_b = ctx.alloc(max_state_h * 12);
    }
    const uint64_t *prev = nullptr;
    uint32_t prev_log = 0;
    for (size_t li = 0; li < launches.size(); li++) {
        merkle::ClassArgs a{};
        a.n_mats = (int)launches[li].idx.size();
        for (int m = 0; m < a.n_mats; m++) {
            a.data[m] = mats[launches[li].idx[m]].d;
            a.width[m] = mats[launches[li].idx[m]].w;
            a.ld[m] = mats[launches[li].idx[m]].w;
        }
        a.log_h = log2u(launches[li].h);
        a.prev = prev;
        a.prev_log_h = prev_log;
        bool last = li + 1 == launches.size();
        uint64_t *out_states = (li % 2 == 0) ? st_a.p : st_b.p;
        a.states_out = last ? nullptr : out_states;
        a.digests_out = last ? t.layers.p : nullptr;
        launch_leaf_class(ctx, a, launches[li].h);
        prev = out_states;
        prev_log = a.log_h;
    }
    finish_tree(ctx, t);
}

}  // namespace p3g
