// AIRs given as symbolic constraint expressions, with a constraint kernel
// generated from them at run time.
//
// The reference is generic over any LiftedAir: it runs the AIR's eval() on a
// SymbolicAirBuilder to learn each constraint's degree and the quotient
// degree (p3-miden-lifted-air/src/air.rs:225-247), on a layout builder to
// split the constraints into base-field and extension-field streams
// (p3-miden-lifted-stark/src/prover/constraints/layout.rs:27-37), and then
// evaluates eval() on every point of the quotient coset gJ with a packed
// folder (constraints/mod.rs:63-179, folder.rs:86-284). Here the caller hands
// over the symbolic form directly — the expression DAG SymbolicAirBuilder
// records, plus the AIR's dimensions and periodic columns — and this file:
//
//   * validates the DAG (operands before their node, variables inside the
//     declared dimensions: the bounds LiftedAir::is_valid_builder checks);
//   * derives the degree multiples and log_quotient_degree
//     (log2_ceil(max(M, 2) - 1)) and the base/extension layout;
//   * types every node (base field unless it reads an aux column, a
//     challenge or an aux value), emits straight-line CUDA for one point of
//     gJ — loads of the used trace cells, the selectors the AIR reads, the
//     DAG in base or extension arithmetic, and the fold
//     sum_k alpha^{K-1-k} C_k with base constraints on a lazy 160-bit
//     accumulator per coordinate (the decompose_alpha form) and extension
//     constraints as extension products — and compiles it with NVRTC for
//     this device (sm_100a), one thread per point;
//   * evaluates the same DAG on the host in the extension field for the
//     verifier's check at the out-of-domain point.
//
// Degree multiples follow p3-air's SymbolicExpression::degree_multiple:
// trace cells and periodic columns 1, is_first_row / is_last_row 1,
// is_transition 0, constants, public values, challenges and aux values 0;
// sums take the maximum, products the sum.
#pragma once
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstring>
#include <mutex>
#include <sstream>
#include <thread>
#include <string>
#include <vector>

#include "context.cuh"
#include "gl.cuh"

namespace sym {

// the text of gl.cuh, embedded at build time (build.py writes gen_gl_src.inc)
static const char *kGlSource =
#include "gen_gl_src.inc"
    ;

enum Op : uint32_t {
    CONST = 0, MAIN = 1, AUX = 2, PUBLIC = 3, RANDOMNESS = 4, AUX_VALUE = 5, PERIODIC = 6,
    IS_FIRST_ROW = 7, IS_LAST_ROW = 8, IS_TRANSITION = 9, ADD = 10, SUB = 11, MUL = 12, NEG = 13
};

struct Node {
    uint32_t op, a, b, pad;
    uint64_t value;
};

struct Desc {
    uint32_t main_width, aux_width, num_randomness, num_aux_values, num_public_values, num_periodic;
    std::vector<uint64_t> periodic_lengths, periodic_values;
    std::vector<Node> nodes;
    std::vector<uint32_t> constraints;
    std::vector<uint8_t> is_ext;
};

// Offsets of the per-call constant block the kernel reads (uniform loads):
// public values, randomness (2 words each), aux values (2 each), alpha
// powers alpha^{K-1-k} (2 each, emission order).
struct KLayout {
    uint64_t pub = 0, rnd = 0, auxv = 0, alpha = 0, words = 0;
};

struct Air {
    Desc d;
    std::vector<uint32_t> degree;   // per node
    std::vector<uint8_t> ext;       // per node: value in the extension field
    uint32_t max_degree = 0, log_qd = 0;
    bool uses_first = false, uses_last = false, uses_trans = false;
    std::vector<uint64_t> base_idx, ext_idx;  // ConstraintLayout
    KLayout kl;
    std::vector<std::vector<uint32_t>> chunks;  // constraint indices of each generated kernel
    size_t chunk_nodes = 500;  // DAG nodes per chunk (a launch-shape choice; every value gives the same sums)
    std::string source, log;
    std::vector<std::vector<char>> cubins;  // one per compiled group of chunks
    std::vector<cudaLibrary_t> libs;
    std::vector<cudaKernel_t> kernels;  // one per chunk: p3g_sym_eval_<c>
    int device = -1;
    ~Air() {
        for (cudaLibrary_t l : libs) cudaLibraryUnload(l);
    }
};

// 0 = valid; otherwise a description of the first problem
inline const char *validate(const Desc &d) {
    const size_t n = d.nodes.size();
    if (d.periodic_lengths.size() != d.num_periodic) return "periodic_lengths size";
    uint64_t total = 0;
    for (uint64_t p : d.periodic_lengths) {
        if (p == 0 || (p & (p - 1)) || p > (1ull << 30)) return "periodic column length not a power of two";
        total += p;
    }
    if (total != d.periodic_values.size()) return "periodic_values size";
    for (uint64_t v : d.periodic_values)
        if (v >= gl::P) return "periodic value not canonical";
    for (size_t i = 0; i < n; i++) {
        const Node &x = d.nodes[i];
        switch (x.op) {
            case CONST: if (x.value >= gl::P) return "constant not canonical"; break;
            case MAIN: if (x.a >= d.main_width || x.b > 1) return "main variable out of range"; break;
            case AUX: if (x.a >= d.aux_width || x.b > 1) return "aux variable out of range"; break;
            case PUBLIC: if (x.a >= d.num_public_values) return "public value out of range"; break;
            case RANDOMNESS: if (x.a >= d.num_randomness) return "randomness out of range"; break;
            case AUX_VALUE: if (x.a >= d.num_aux_values) return "aux value out of range"; break;
            case PERIODIC: if (x.a >= d.num_periodic) return "periodic column out of range"; break;
            case IS_FIRST_ROW: case IS_LAST_ROW: case IS_TRANSITION: break;
            case ADD: case SUB: case MUL: if (x.a >= i || x.b >= i) return "operand after its node"; break;
            case NEG: if (x.a >= i) return "operand after its node"; break;
            default: return "unknown node kind";
        }
    }
    if (d.constraints.size() != d.is_ext.size()) return "is_ext size";
    for (uint32_t c : d.constraints)
        if (c >= n) return "constraint node out of range";
    if (d.aux_width == 0) return "aux_width must be positive (LiftedAir::validate)";
    return nullptr;
}

inline void analyse(Air &A) {
    const Desc &d = A.d;
    const size_t n = d.nodes.size();
    A.degree.assign(n, 0);
    A.ext.assign(n, 0);
    for (size_t i = 0; i < n; i++) {
        const Node &x = d.nodes[i];
        uint32_t &g = A.degree[i];
        uint8_t &e = A.ext[i];
        switch (x.op) {
            case MAIN: case PERIODIC: g = 1; break;
            case AUX: g = 1, e = 1; break;
            case IS_FIRST_ROW: case IS_LAST_ROW: g = 1; break;
            case RANDOMNESS: case AUX_VALUE: e = 1; break;
            case ADD: case SUB:
                g = std::max(A.degree[x.a], A.degree[x.b]);
                e = A.ext[x.a] | A.ext[x.b];
                break;
            case MUL:
                g = A.degree[x.a] + A.degree[x.b];
                e = A.ext[x.a] | A.ext[x.b];
                break;
            case NEG: g = A.degree[x.a], e = A.ext[x.a]; break;
            default: break;
        }
    }
    A.max_degree = 0;
    for (uint32_t c : d.constraints) A.max_degree = std::max(A.max_degree, A.degree[c]);
    uint32_t m = std::max<uint32_t>(A.max_degree, 2);
    A.log_qd = 0;
    while ((1u << A.log_qd) < m - 1) A.log_qd++;
    A.base_idx.clear();
    A.ext_idx.clear();
    for (size_t k = 0; k < d.constraints.size(); k++) (d.is_ext[k] ? A.ext_idx : A.base_idx).push_back(k);
    // only nodes reachable from a constraint are emitted
    std::vector<uint8_t> live(n, 0);
    for (uint32_t c : d.constraints) live[c] = 1;
    for (size_t i = n; i-- > 0;) {
        if (!live[i]) continue;
        const Node &x = d.nodes[i];
        if (x.op == ADD || x.op == SUB || x.op == MUL) live[x.a] = live[x.b] = 1;
        if (x.op == NEG) live[x.a] = 1;
        if (x.op == IS_FIRST_ROW) A.uses_first = true;
        if (x.op == IS_LAST_ROW) A.uses_last = true;
        if (x.op == IS_TRANSITION) A.uses_trans = true;
    }
    KLayout &k = A.kl;
    k.pub = 0;
    k.rnd = k.pub + d.num_public_values;
    k.auxv = k.rnd + 2ull * d.num_randomness;
    k.alpha = k.auxv + 2ull * d.num_aux_values;
    k.words = k.alpha + 2ull * d.constraints.size();
}

// Arguments of the generated kernel (the same layout is declared in the
// generated source).
struct KArgs {
    // the first qh rows (the quotient domain gJ, bit-reversed) of the main
    // and aux LDEs, column-major: cell (row r, word c) at [c * qh + r]; the
    // aux trace has 2 words per EF column
    const uint64_t *main;
    uint64_t main_w;
    const uint64_t *aux;
    uint64_t aux_w2;
    const uint64_t *per;   // periodic LDE on gJ, natural order
    uint64_t per_h, per_w;
    const uint64_t *k;     // constant block (KLayout)
    uint64_t qh;
    uint32_t log_qh, pad0;
    uint64_t D;
    uint64_t shift;        // coset shift of this trace
    const uint64_t *wq_lo, *wq_hi;  // two-level table of w_{qh}^e
    uint32_t wq_lo_bits, pad1;
    uint64_t omega_h_inv;
    uint64_t zh[8];        // Z_H on gJ, period D
    uint64_t *acc;         // EF accumulator, += the folded numerator
};

// Constraints are split into chunks of bounded code size (at most
// A.chunk_nodes DAG nodes each, shared subexpressions counted once per chunk);
// each chunk is one kernel that adds its part of the fold into acc. The fold
// is linear, so launching the chunks one after another on the same stream
// gives the same sum. A small AIR is one chunk.

inline void split_chunks(Air &A) {
    const Desc &d = A.d;
    const size_t n = d.nodes.size();
    A.chunks.assign(1, {});
    std::vector<uint32_t> owner(n, 0), seen(n, 0), st, walk;
    uint32_t cid = 1, epoch = 0;
    size_t in_chunk = 0;
    // the nodes under `root` that the current chunk does not hold yet
    auto collect = [&](uint32_t root) {
        walk.clear();
        st.assign(1, root);
        ++epoch;
        while (!st.empty()) {
            const uint32_t i = st.back();
            st.pop_back();
            if (owner[i] == cid || seen[i] == epoch) continue;
            seen[i] = epoch;
            walk.push_back(i);
            const Node &x = d.nodes[i];
            if (x.op == ADD || x.op == SUB || x.op == MUL) st.push_back(x.a), st.push_back(x.b);
            if (x.op == NEG) st.push_back(x.a);
        }
    };
    for (size_t k = 0; k < d.constraints.size(); k++) {
        collect(d.constraints[k]);
        if (!A.chunks.back().empty() && in_chunk + walk.size() > A.chunk_nodes) {
            A.chunks.emplace_back();
            cid++;
            in_chunk = 0;
            collect(d.constraints[k]);
        }
        for (uint32_t i : walk) owner[i] = cid;
        in_chunk += walk.size();
        A.chunks.back().push_back((uint32_t)k);
    }
}

// The source of the kernels of chunks [c0, c1): the field arithmetic
// (gl.cuh), the argument block and one kernel per chunk.
inline std::string generate_range(const Air &A, size_t c0, size_t c1) {
    const Desc &d = A.d;
    std::ostringstream o;
    o << "// generated by libp3miden_b200 (symair.cuh) from a symbolic AIR: " << d.nodes.size() << " nodes, "
      << d.constraints.size() << " constraints in " << A.chunks.size() << " kernels (here " << c0 << ".." << c1
      << "), max degree " << A.max_degree << "\n";
    o << kGlSource << "\n";
    o << R"K(
struct KArgs {
    const uint64_t *main; uint64_t main_w;
    const uint64_t *aux; uint64_t aux_w2;
    const uint64_t *per; uint64_t per_h, per_w;
    const uint64_t *k;
    uint64_t qh; uint32_t log_qh, pad0; uint64_t D;
    uint64_t shift;
    const uint64_t *wq_lo, *wq_hi; uint32_t wq_lo_bits, pad1;
    uint64_t omega_h_inv;
    uint64_t zh[8];
    uint64_t *acc;
};
)K";
    const size_t n = d.nodes.size();
    auto as_ef = [&](uint32_t j) {
        std::string v = "v" + std::to_string(j);
        return A.ext[j] ? v : "gl::ef{" + v + ", 0}";
    };
    // Two rewrites over the whole DAG (a node's readers can sit in any chunk):
    // a base product read only by products (and the fold, which takes any
    // value below 2^64) keeps its weakly reduced value, without the canonical
    // step; a base (a + b) - (c + c) whose two inner sums have no other reader
    // (the XOR of bits, a + b - 2ab) is emitted as (a - c) + (b - c).
    std::vector<uint32_t> n_users(n, 0);
    std::vector<uint8_t> only_mul(n, 1), is_root(n, 0), weak(n, 0), fused(n, 0);
    for (uint32_t c : d.constraints) is_root[c] = 1;
    for (size_t i = 0; i < n; i++) {
        const Node &x = d.nodes[i];
        auto use = [&](uint32_t j) {
            n_users[j]++;
            if (x.op != MUL) only_mul[j] = 0;
        };
        if (x.op == ADD || x.op == SUB || x.op == MUL) use(x.a), use(x.b);
        if (x.op == NEG) use(x.a);
    }
    for (size_t i = 0; i < n; i++) {
        const Node &x = d.nodes[i];
        if (A.ext[i]) continue;
        if (x.op == MUL && only_mul[i]) weak[i] = 1;
        if (x.op == SUB && x.a != x.b) {
            const Node &sa = d.nodes[x.a], &sb = d.nodes[x.b];
            fused[i] = sa.op == ADD && sb.op == ADD && sb.a == sb.b && !A.ext[x.a] && !A.ext[x.b] &&
                       n_users[x.a] == 1 && n_users[x.b] == 1 && !is_root[x.a] && !is_root[x.b];
        }
    }
    // A third: a chain of sums and differences whose inner links each have one
    // reader, itself a link (such as the Horner recombination of a limb from
    // its bits, acc + acc + bit), is accumulated as a Wide and reduced once at
    // the chain's end (inner[i]: i is such a link).
    std::vector<uint8_t> linear(n, 0), inner(n, 0);
    std::vector<int64_t> reader(n, -1);  // the one node reading i, -1 for none, -2 for several
    for (size_t i = 0; i < n; i++) {
        const Node &x = d.nodes[i];
        linear[i] = !A.ext[i] && !fused[i] && (x.op == ADD || x.op == SUB || x.op == NEG);
        auto read = [&](uint32_t j) { reader[j] = reader[j] == -1 || reader[j] == (int64_t)i ? (int64_t)i : -2; };
        if (x.op == ADD || x.op == SUB || x.op == MUL) read(x.a), read(x.b);
        if (x.op == NEG) read(x.a);
    }
    for (size_t i = 0; i < n; i++)
        inner[i] = linear[i] && !is_root[i] && reader[i] >= 0 && linear[reader[i]];
    std::vector<uint8_t> live(n);
    for (size_t c = c0; c < c1; c++) {
        const std::vector<uint32_t> &ks = A.chunks[c];
        std::fill(live.begin(), live.end(), 0);
        for (uint32_t k : ks) live[d.constraints[k]] = 1;
        bool first = false, last = false, trans = false;
        for (size_t i = n; i-- > 0;) {
            if (!live[i]) continue;
            const Node &x = d.nodes[i];
            if (x.op == ADD || x.op == SUB || x.op == MUL) live[x.a] = live[x.b] = 1;
            if (x.op == NEG) live[x.a] = 1;
            first |= x.op == IS_FIRST_ROW, last |= x.op == IS_LAST_ROW, trans |= x.op == IS_TRANSITION;
        }
        o << "extern \"C\" __global__ void __launch_bounds__(128) p3g_sym_eval_" << c
          << "(const __grid_constant__ KArgs a) {\n";
        // thread r reads storage row r (point m = bitrev(r)) and the row of
        // the point m + D: a warp's 32 rows, and its 32 next rows, each lie in
        // one aligned 32-row block, so every column load is one 256-byte run
        o << R"K(    const uint64_t rl = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (rl >= a.qh) return;
    const uint32_t lq = a.log_qh;
    const uint64_t m = gl::bitrev(rl, lq), rn = gl::bitrev((m + a.D) & (a.qh - 1), lq);
    const uint64_t *ML = a.main + rl, *MN = a.main + rn;
    const uint64_t *AL = a.aux ? a.aux + rl : a.aux, *AN = a.aux ? a.aux + rn : a.aux;
    const uint64_t *PR = a.per ? a.per + (m % a.per_h) * a.per_w : a.per;
    const uint64_t *K = a.k;
    (void)ML; (void)MN; (void)AL; (void)AN; (void)PR; (void)K; (void)lq;
)K";
        if (first || last || trans) {
            o << "    const uint64_t mlo = m & ((1ull << a.wq_lo_bits) - 1), mhi = m >> a.wq_lo_bits;\n"
                 "    uint64_t wm = __ldg(a.wq_lo + mlo);\n"
                 "    if (mhi) wm = gl::mul(wm, __ldg(a.wq_hi + mhi));\n"
                 "    const uint64_t x = gl::mul(a.shift, wm);\n";
            if (first || last) o << "    const uint64_t zh = a.zh[m & (a.D - 1)];\n";
            if (first) o << "    const uint64_t s_first = gl::mul(zh, gl::inv(gl::sub(x, 1)));\n";
            if (last) o << "    const uint64_t s_last = gl::mul(zh, gl::inv(gl::sub(x, a.omega_h_inv)));\n";
            if (trans) o << "    const uint64_t s_trans = gl::sub(x, a.omega_h_inv);\n";
        }
        // constraint by constraint: the nodes of its expression not emitted
        // yet, in post-order (each load just before its first use), then its
        // term of the fold, so that a value lives only while a later node of
        // the chunk still reads it (register pressure sets the occupancy of
        // these long straight-line kernels). Base constraints go into two lazy
        // accumulators (one per coordinate of alpha^{K-1-k}), extension
        // constraints into an extension sum.
        std::vector<uint8_t> done(n, 0);
        std::vector<std::pair<uint32_t, bool>> st;
        std::vector<uint8_t> bits(n, 64);
        // a multiple of p at or above 2^b (64 <= b <= 95), as "lo, hi"
        auto p_multiple = [](unsigned b) {
            const unsigned __int128 c = (unsigned __int128)gl::P << (b - 63);  // p * 2^t > 2^(63 + t)
            return std::to_string((uint64_t)c) + "ull, " + std::to_string((uint32_t)(c >> 64)) + "u";
        };
        // a chain link or the end of a chain: Wide arithmetic on its operands
        auto emit_wide = [&](size_t i) -> bool {
            const Node &x = d.nodes[i];
            if (!linear[i] || !(inner[x.a] || (x.op != NEG && inner[x.b]) || inner[i])) return false;
            auto operand = [&](uint32_t j, unsigned &b) -> std::string {
                if (inner[j]) {
                    b = bits[j];
                    return "w" + std::to_string(j);
                }
                b = 64;
                return "gl::Wide{v" + std::to_string(j) + ", 0}";
            };
            unsigned ba = 64, bb = 64, nb;
            std::string ea = operand(x.a, ba), eb = x.op == NEG ? "" : operand(x.b, bb);
            nb = x.op == ADD ? std::max(ba, bb) + 1 : x.op == SUB ? std::max(ba, bb + 1) + 1 : ba + 1;
            if (nb > 95) {  // close the operands' chains here (each is read by this node only)
                for (uint32_t j : {x.a, x.b}) {
                    if (x.op == NEG && j == x.b) continue;
                    if (inner[j] && bits[j] > 64) {
                        o << "    const uint64_t v" << j << " = gl::wide_canon(w" << j << ");\n";
                        inner[j] = 0;
                    }
                }
                ea = operand(x.a, ba);
                if (x.op != NEG) eb = operand(x.b, bb);
                nb = x.op == ADD ? std::max(ba, bb) + 1 : x.op == SUB ? std::max(ba, bb + 1) + 1 : ba + 1;
            }
            std::string rhs = x.op == ADD   ? "gl::wide_add(" + ea + ", " + eb + ")"
                              : x.op == SUB ? "gl::wide_sub(" + ea + ", " + eb + ", " + p_multiple(bb) + ")"
                                            : "gl::wide_neg(" + ea + ", " + p_multiple(ba) + ")";
            if (inner[i]) {
                o << "    const gl::Wide w" << i << " = " << rhs << ";\n";
                bits[i] = (uint8_t)nb;
            } else {
                o << "    const uint64_t v" << i << " = gl::wide_canon(" << rhs << ");\n";
            }
            return true;
        };
        auto emit_node = [&](size_t i) {
            if (emit_wide(i)) return;
            const Node &x = d.nodes[i];
            const std::string v = "v" + std::to_string(i);
            const char *ty = A.ext[i] ? "const gl::ef " : "const uint64_t ";
            o << "    " << ty << v << " = ";
            switch (x.op) {
                case CONST: o << x.value << "ull"; break;
                case MAIN: o << "__ldg(" << (x.b ? "MN" : "ML") << " + (" << x.a << "ull << lq))"; break;
                case AUX:
                    o << "gl::ef{__ldg(" << (x.b ? "AN" : "AL") << " + (" << 2 * x.a << "ull << lq)), __ldg("
                      << (x.b ? "AN" : "AL") << " + (" << 2 * x.a + 1 << "ull << lq))}";
                    break;
                case PUBLIC: o << "__ldg(K + " << A.kl.pub + x.a << ")"; break;
                case RANDOMNESS:
                    o << "gl::ef{__ldg(K + " << A.kl.rnd + 2 * x.a << "), __ldg(K + " << A.kl.rnd + 2 * x.a + 1 << ")}";
                    break;
                case AUX_VALUE:
                    o << "gl::ef{__ldg(K + " << A.kl.auxv + 2 * x.a << "), __ldg(K + " << A.kl.auxv + 2 * x.a + 1
                      << ")}";
                    break;
                case PERIODIC: o << "__ldg(PR + " << x.a << ")"; break;
                case IS_FIRST_ROW: o << "s_first"; break;
                case IS_LAST_ROW: o << "s_last"; break;
                case IS_TRANSITION: o << "s_trans"; break;
                case ADD: case SUB: {
                    const char *f = x.op == ADD ? "add" : "sub";
                    if (fused[i]) {
                        const uint32_t a = d.nodes[x.a].a, b = d.nodes[x.a].b, c = d.nodes[x.b].a;
                        o << "gl::add(gl::sub(v" << a << ", v" << c << "), gl::sub(v" << b << ", v" << c << "))";
                    } else if (A.ext[i]) o << "gl::ef_" << f << "(" << as_ef(x.a) << ", " << as_ef(x.b) << ")";
                    else o << "gl::" << f << "(v" << x.a << ", v" << x.b << ")";
                    break;
                }
                case MUL:
                    if (!A.ext[i]) o << (weak[i] ? "gl::mul_weak(v" : "gl::mul(v") << x.a << ", v" << x.b << ")";
                    else if (!A.ext[x.a]) o << "gl::ef_mulf(v" << x.b << ", v" << x.a << ")";
                    else if (!A.ext[x.b]) o << "gl::ef_mulf(v" << x.a << ", v" << x.b << ")";
                    else o << "gl::ef_mul(v" << x.a << ", v" << x.b << ")";
                    break;
                default:  // NEG
                    o << (A.ext[i] ? "gl::ef_neg(v" : "gl::neg(v") << x.a << ")";
                    break;
            }
            o << ";\n";
        };
        o << "    gl::Acc f0, f1;\n    gl::ef fe = gl::ef_zero();\n";
        for (uint32_t k : ks) {
            const uint32_t cn = d.constraints[k];
            st.assign(1, {cn, false});
            while (!st.empty()) {  // iterative post-order over the nodes not emitted yet
                const auto [i, expanded] = st.back();
                st.pop_back();
                if (done[i]) continue;
                const Node &x = d.nodes[i];
                const bool binary = x.op == ADD || x.op == SUB || x.op == MUL;
                if (!expanded && (binary || x.op == NEG)) {
                    st.push_back({i, true});
                    if (fused[i]) {  // (a + b) - (c + c): the inner sums are not emitted
                        st.push_back({d.nodes[x.b].a, false});
                        st.push_back({d.nodes[x.a].b, false});
                        st.push_back({d.nodes[x.a].a, false});
                        continue;
                    }
                    if (binary) st.push_back({x.b, false});
                    st.push_back({x.a, false});
                    continue;
                }
                done[i] = 1;
                emit_node(i);
            }
            const uint64_t ap = A.kl.alpha + 2ull * k;
            if (!A.ext[cn])
                o << "    f0.mac(v" << cn << ", __ldg(K + " << ap << ")); f1.mac(v" << cn << ", __ldg(K + " << ap + 1
                  << "));\n";
            else
                o << "    fe = gl::ef_add(fe, gl::ef_mul(v" << cn << ", gl::ef{__ldg(K + " << ap << "), __ldg(K + "
                  << ap + 1 << ")}));\n";
        }
        o << R"K(    const gl::ef r = gl::ef_add(gl::ef{f0.reduce(), f1.reduce()}, fe);
    uint64_t *out = a.acc + 2 * m;
    out[0] = gl::add(out[0], r.c0);
    out[1] = gl::add(out[1], r.c1);
}
)K";
    }
    return o.str();
}

// The whole generated program (every chunk's kernel); splits the chunks.
inline std::string generate(Air &A) {
    split_chunks(A);
    return generate_range(A, 0, A.chunks.size());
}

struct CompileError {
    std::string what;
};

// NVRTC: source -> cubin for sm_<cc> (the architecture-specific target, like
// the library itself). No device is needed. Throws with the compiler log.
inline void nvrtc_cubin(const std::string &source, int cc, std::vector<char> &cubin, std::string &log) {
    const std::string arch = "--gpu-architecture=sm_" + std::to_string(cc) + (cc >= 90 ? "a" : "");
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, source.c_str(), "p3g_sym_eval.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        throw p3g::CudaError{p3g::ERR_CUDA, "nvrtcCreateProgram failed"};
    const char *opts[] = {arch.c_str(), "--std=c++17", "-default-device"};
    nvrtcResult r = nvrtcCompileProgram(prog, 3, opts);
    size_t log_n = 0;
    nvrtcGetProgramLogSize(prog, &log_n);
    log.assign(log_n, '\0');
    if (log_n) nvrtcGetProgramLog(prog, &log[0]);
    if (r != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        throw p3g::CudaError{p3g::ERR_CUDA, "generated constraint kernel failed to compile: " + log.substr(0, 2000)};
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    cubin.resize(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
}

// Compile the chunks in groups, one NVRTC program per group, on up to one
// host thread per core (compile time grows faster than linearly in the size
// of a straight-line kernel, and groups compile independently).
inline void compile_cubins(Air &A, int cc) {
    const size_t nch = A.chunks.size();
    unsigned hw = std::thread::hardware_concurrency();
    const size_t groups = std::max<size_t>(1, std::min<size_t>(nch, hw ? hw : 4));
    A.cubins.assign(groups, {});
    std::vector<std::string> logs(groups);
    std::vector<std::string> errs(groups);
    std::vector<std::thread> th;
    for (size_t g = 0; g < groups; g++)
        th.emplace_back([&, g] {
            const size_t c0 = nch * g / groups, c1 = nch * (g + 1) / groups;
            try {
                nvrtc_cubin(generate_range(A, c0, c1), cc, A.cubins[g], logs[g]);
            } catch (const p3g::CudaError &e) {
                errs[g] = e.what;
            }
        });
    for (auto &t : th) t.join();
    for (size_t g = 0; g < groups; g++)
        if (!errs[g].empty()) throw p3g::CudaError{p3g::ERR_CUDA, errs[g]};
    A.log = logs[0];
}

inline void compile(Air &A, int device) {
    int major = 0, minor = 0;
    CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    CK(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
    compile_cubins(A, major * 10 + minor);
    const size_t nch = A.chunks.size(), groups = A.cubins.size();
    A.kernels.resize(nch);
    for (size_t g = 0; g < groups; g++) {
        cudaLibrary_t lib = nullptr;
        CK(cudaLibraryLoadData(&lib, A.cubins[g].data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        A.libs.push_back(lib);
        for (size_t c = nch * g / groups; c < nch * (g + 1) / groups; c++) {
            CK(cudaLibraryGetKernel(&A.kernels[c], lib, ("p3g_sym_eval_" + std::to_string(c)).c_str()));
            // load the kernel into the device's context now rather than at its
            // first launch (lazy loading would put it inside the first proof)
            cudaFuncAttributes attr;
            CK(cudaFuncGetAttributes(&attr, (const void *)A.kernels[c]));
        }
    }
    A.device = device;
}

// Host evaluation of every constraint at one point, all in the extension
// field (base values embedded): the verifier's ConstraintFolder at z
// (p3-miden-lifted-stark/src/verifier/mod.rs:286-339).
struct Point {
    const gl::ef *main_local, *main_next, *aux_local, *aux_next;
    const uint64_t *pub;
    const gl::ef *rand, *auxv, *periodic;
    gl::ef sel[3];
};
inline gl::ef fold_at(const Air &A, const Point &pt, gl::ef alpha) {
    const Desc &d = A.d;
    std::vector<gl::ef> v(d.nodes.size());
    for (size_t i = 0; i < d.nodes.size(); i++) {
        const Node &x = d.nodes[i];
        gl::ef r;
        switch (x.op) {
            case CONST: r = gl::ef{x.value, 0}; break;
            case MAIN: r = x.b ? pt.main_next[x.a] : pt.main_local[x.a]; break;
            case AUX: r = x.b ? pt.aux_next[x.a] : pt.aux_local[x.a]; break;
            case PUBLIC: r = gl::ef{pt.pub[x.a], 0}; break;
            case RANDOMNESS: r = pt.rand[x.a]; break;
            case AUX_VALUE: r = pt.auxv[x.a]; break;
            case PERIODIC: r = pt.periodic[x.a]; break;
            case IS_FIRST_ROW: r = pt.sel[0]; break;
            case IS_LAST_ROW: r = pt.sel[1]; break;
            case IS_TRANSITION: r = pt.sel[2]; break;
            case ADD: r = gl::ef_add(v[x.a], v[x.b]); break;
            case SUB: r = gl::ef_sub(v[x.a], v[x.b]); break;
            case MUL: r = gl::ef_mul(v[x.a], v[x.b]); break;
            default: r = gl::ef_neg(v[x.a]); break;
        }
        v[i] = r;
    }
    gl::ef f = gl::ef_zero();
    for (uint32_t c : d.constraints) f = gl::ef_add(gl::ef_mul(f, alpha), v[c]);
    return f;
}

// The periodic columns repeated to the largest period (max_p x num_periodic,
// row-major): LiftedAir::periodic_columns_matrix (air.rs:64-84).
inline std::vector<uint64_t> periodic_matrix(const Desc &d, uint64_t &max_p) {
    max_p = 0;
    for (uint64_t p : d.periodic_lengths) max_p = std::max(max_p, p);
    std::vector<uint64_t> m(max_p * d.num_periodic);
    uint64_t off = 0;
    for (uint32_t c = 0; c < d.num_periodic; c++) {
        const uint64_t p = d.periodic_lengths[c];
        for (uint64_t r = 0; r < max_p; r++) m[r * d.num_periodic + c] = d.periodic_values[off + r % p];
        off += p;
    }
    return m;
}

// PeriodicPolys::eval_at (p3-miden-lifted-stark/src/verifier/periodic.rs:31-80):
// column c's interpolant on the subgroup of order p, at z^(max_h / p).
inline void periodic_at(const Desc &d, uint64_t max_h, gl::ef z, std::vector<gl::ef> &out) {
    out.assign(d.num_periodic, gl::ef_zero());
    uint64_t off = 0;
    for (uint32_t c = 0; c < d.num_periodic; c++) {
        const uint64_t p = d.periodic_lengths[c];
        uint32_t lp = 0;
        while ((1ull << lp) < p) lp++;
        const uint64_t winv = gl::inv(gl::root(lp)), pinv = gl::inv(p % gl::P);
        std::vector<uint64_t> coef(p);
        for (uint64_t k = 0; k < p; k++) {  // inverse DFT (NaiveDft::idft)
            uint64_t s = 0, wk = gl::pow(winv, k), x = 1;
            for (uint64_t j = 0; j < p; j++) s = gl::add(s, gl::mul(d.periodic_values[off + j], x)), x = gl::mul(x, wk);
            coef[k] = gl::mul(s, pinv);
        }
        const gl::ef y = gl::ef_pow(z, max_h / p);
        gl::ef acc = gl::ef_zero();
        for (uint64_t k = p; k-- > 0;) acc = gl::ef_add(gl::ef_mul(acc, y), gl::ef{coef[k], 0});
        out[c] = acc;
        off += p;
    }
}

}  // namespace sym
