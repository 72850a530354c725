// Host-side Fiat-Shamir transcript: ProverTranscript over a duplex
// challenger (p3-miden-transcript/src/prover.rs:15-178; challenger semantics
// of DuplexChallenger<F, Poseidon2, 12, 8>):
//  observe: clear buffered outputs, buffer the input, duplex at 8 inputs;
//  sample: duplex if inputs are pending or outputs exhausted, pop the last
//          output word;
//  duplex: overwrite state[0..k] with the k pending inputs, permute,
//          outputs = state[0..8];
//  send_* records and observes, hint_* records only, grind records the
//  witness; finalize = one more duplex, digest = the 12-word state.
#pragma once
#include <vector>

#include "gl.cuh"
#include "poseidon2.cuh"

namespace p3g {

struct Challenger {
    const uint64_t *p2 = nullptr;
    uint64_t state[12] = {0};
    uint64_t in[8] = {0};
    uint64_t out[8] = {0};
    int n_in = 0, n_out = 0;

    void duplex() {
        for (int i = 0; i < n_in; i++) state[i] = in[i];
        n_in = 0;
        p2::host::permute(state, p2);
        for (int i = 0; i < 8; i++) out[i] = state[i];
        n_out = 8;
    }
    void observe(uint64_t x) {
        n_out = 0;
        in[n_in++] = x;
        if (n_in == 8) duplex();
    }
    uint64_t sample() {
        if (n_in > 0 || n_out == 0) duplex();
        return out[--n_out];
    }
    uint64_t sample_bits(unsigned bits) {
        uint64_t v = sample();
        return bits >= 64 ? v : (v & ((1ull << bits) - 1));
    }
    gl::ef sample_ef() {
        uint64_t a = sample();
        uint64_t b = sample();
        return gl::ef{a, b};
    }
    // would observing w and sampling `bits` bits give zero?
    bool check_witness(unsigned bits, uint64_t w) const {
        Challenger c = *this;
        c.observe(w);
        return c.sample_bits(bits) == 0;
    }
};

struct Transcript {
    Challenger ch;
    std::vector<uint64_t> fields;
    std::vector<uint64_t> commits;

    explicit Transcript(const uint64_t *p2) { ch.p2 = p2; }
    void send_field(uint64_t v) {
        fields.push_back(v);
        ch.observe(v);
    }
    void send_ef(gl::ef v) {
        send_field(v.c0);
        send_field(v.c1);
    }
    void send_commit(const uint64_t *d) {
        for (int i = 0; i < 4; i++) commits.push_back(d[i]);
        for (int i = 0; i < 4; i++) ch.observe(d[i]);
    }
    void hint_field(uint64_t v) { fields.push_back(v); }
    void hint_commit(const uint64_t *d) {
        for (int i = 0; i < 4; i++) commits.push_back(d[i]);
    }
    void finalize(uint64_t digest[12]) {
        ch.duplex();
        for (int i = 0; i < 12; i++) digest[i] = ch.state[i];
    }
};

}  // namespace p3g
