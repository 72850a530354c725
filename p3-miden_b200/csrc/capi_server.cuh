// C-ABI of the batched / serving prover (declarations: include/p3g.h).
#pragma once
#include <memory>
#include <unordered_map>

#include "capi_prove.cuh"
#include "server.cuh"

struct p3g_job_c {
    p3g_pcs_params_c pcs;
    const p3g_instance_c *instances;
    uint64_t n_instances;
    double arrival_s;
};
struct p3g_job_result_c {
    int32_t status;
    int32_t verdict;  // self-check verdict, -1 when not checked
    p3g_proof_c proof;
    double submit_s, start_s, end_s;
    double verify_ms;
};

struct p3g_server {
    std::unique_ptr<p3g::Server> s;
    std::mutex mu;
    std::unordered_map<uint64_t, std::unique_ptr<p3g::ServerJob>> jobs;
    uint64_t next = 1;
    int device = 0;
};

namespace p3g {
inline void fill_proof(const ProofOut &po, p3g_proof_c *out) {
    out->n_fields = po.fields.size();
    out->n_commits = po.commits.size() / 4;
    out->fields = (uint64_t *)malloc(std::max<size_t>(1, po.fields.size()) * 8);
    out->commits = (uint64_t *)malloc(std::max<size_t>(1, po.commits.size()) * 8);
    if (!out->fields || !out->commits) throw std::bad_alloc();
    memcpy(out->fields, po.fields.data(), po.fields.size() * 8);
    memcpy(out->commits, po.commits.data(), po.commits.size() * 8);
    memcpy(out->digest, po.digest, sizeof(po.digest));
    for (int s = 0; s < 12; s++) out->stage_ms[s] = po.stage_ms[s];
    out->gpu_launches = po.launches;
    out->h2d_bytes = po.h2d;
    out->d2h_bytes = po.d2h;
}
inline std::unique_ptr<ServerJob> make_job(const p3g_job_c &j) {
    auto job = std::make_unique<ServerJob>();
    job->pcs = PcsParams{j.pcs.log_blowup,    j.pcs.log_folding_arity, j.pcs.log_final_degree, j.pcs.folding_pow_bits,
                         j.pcs.deep_pow_bits, j.pcs.num_queries,       j.pcs.query_pow_bits};
    for (uint64_t i = 0; i < j.n_instances; i++) {
        const p3g_instance_c &I = j.instances[i];
        job->inst.push_back(to_instance(I));
    }
    job->arrival_s = j.arrival_s;
    return job;
}
inline void fill_result(const ServerJob &job, p3g_job_result_c *r) {
    memset(r, 0, sizeof(*r));
    r->status = job.status;
    r->verdict = job.verdict;
    r->verify_ms = job.verify_ms;
    r->submit_s = job.submit_s;
    r->start_s = job.start_s;
    r->end_s = job.end_s;
    if (job.status == OK) fill_proof(job.out, &r->proof);
}
}  // namespace p3g

P3G_API int p3g_server_create(int device, const uint64_t *poseidon2_params130, uint32_t n_workers,
                              uint64_t hbm_budget_bytes, p3g_server **out) {
    if (!out || !poseidon2_params130 || n_workers == 0 || n_workers > 64) return p3g::ERR_INVALID;
    *out = nullptr;
    auto *srv = new p3g_server();
    try {
        CK(cudaSetDevice(device));
        p3g::ensure_keccak_tables(device);
        srv->device = device;
        srv->s = std::make_unique<p3g::Server>(device, poseidon2_params130, n_workers, hbm_budget_bytes);
    } catch (const p3g::CudaError &e) {
        delete srv;
        return e.status;
    }
    *out = srv;
    return p3g::OK;
}

P3G_API void p3g_server_destroy(p3g_server *srv) {
    if (!srv) return;
    if (srv->s) srv->s->wait_all();
    srv->s.reset();
    delete srv;
}

// Enqueue a job now (its arrival_s is ignored); traces stay borrowed until
// p3g_server_wait returns for the ticket.
P3G_API int p3g_server_set_self_check(p3g_server *srv, int32_t enabled) {
    if (!srv) return p3g::ERR_INVALID;
    srv->s->set_self_check(enabled != 0);
    return p3g::OK;
}

// Saved launch shapes (p3g_ctx_set_lde_split / p3g_ctx_set_slab_columns) for
// every worker of the server; call before submitting jobs.
P3G_API int p3g_server_set_lde_split(p3g_server *srv, uint32_t log_height, const uint32_t *sizes, uint32_t n) {
    if (!srv || (n && !sizes)) return p3g::ERR_INVALID;
    std::vector<uint32_t> v(sizes, sizes + n);
    if (n && !p3g::valid_split(log_height, v)) return p3g::ERR_INVALID;
    srv->s->set_lde_split(log_height, v);
    return p3g::OK;
}
P3G_API int p3g_server_set_slab_columns(p3g_server *srv, uint64_t cols) {
    if (!srv || (cols % 8) != 0) return p3g::ERR_INVALID;
    srv->s->set_slab_columns(cols);
    return p3g::OK;
}

// At most n heavy jobs (LDEs above 2^26 words) at a time; 0 lifts the limit.
P3G_API int p3g_server_set_max_heavy(p3g_server *srv, uint32_t n) {
    if (!srv) return p3g::ERR_INVALID;
    srv->s->set_max_heavy(n);
    return p3g::OK;
}

P3G_API int p3g_server_submit(p3g_server *srv, const p3g_job_c *job, uint64_t *ticket) {
    if (!srv || !job || !ticket) return p3g::ERR_INVALID;
    int v = p3g::validate(&job->pcs, job->instances, job->n_instances);
    if (v != p3g::OK) return v;
    auto j = p3g::make_job(*job);
    p3g::ServerJob *raw = j.get();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        *ticket = srv->next++;
        srv->jobs[*ticket] = std::move(j);
    }
    srv->s->submit(raw);
    return p3g::OK;
}

// Block until the ticket's job finished; the proof buffers are malloc'ed
// (release with p3g_proof_free). Returns the job's status.
P3G_API int p3g_server_wait(p3g_server *srv, uint64_t ticket, p3g_job_result_c *out) {
    if (!srv || !out) return p3g::ERR_INVALID;
    std::unique_ptr<p3g::ServerJob> job;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->jobs.find(ticket);
        if (it == srv->jobs.end()) return p3g::ERR_INVALID;
        job = std::move(it->second);
        srv->jobs.erase(it);
    }
    srv->s->wait(job.get());
    try {
        p3g::fill_result(*job, out);
    } catch (const std::bad_alloc &) {
        return p3g::ERR_OOM;
    }
    return job->status;
}

// Serve a list of jobs: each is submitted when arrival_s seconds have passed
// since the call started (all 0 = one batch), then all are awaited.
// results[i].status holds each job's own status; returns P3G_OK unless an
// argument is invalid.
P3G_API int p3g_server_run(p3g_server *srv, const p3g_job_c *jobs, uint64_t n, p3g_job_result_c *results) {
    if (!srv || (!jobs && n) || (!results && n)) return p3g::ERR_INVALID;
    std::vector<std::unique_ptr<p3g::ServerJob>> js(n);
    std::vector<int> invalid(n, p3g::OK);
    for (uint64_t i = 0; i < n; i++) {
        invalid[i] = p3g::validate(&jobs[i].pcs, jobs[i].instances, jobs[i].n_instances);
        if (invalid[i] == p3g::OK) js[i] = p3g::make_job(jobs[i]);
    }
    // submission order = arrival order
    std::vector<uint64_t> order(n);
    for (uint64_t i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return jobs[a].arrival_s < jobs[b].arrival_s; });
    const double t0 = srv->s->now_s();
    for (uint64_t i : order) {
        if (!js[i]) continue;
        double target = t0 + jobs[i].arrival_s;
        double now = srv->s->now_s();
        if (target > now) std::this_thread::sleep_for(std::chrono::duration<double>(target - now));
        srv->s->submit(js[i].get());
    }
    srv->s->wait_all();
    for (uint64_t i = 0; i < n; i++) {
        if (!js[i]) {
            memset(&results[i], 0, sizeof(results[i]));
            results[i].status = invalid[i];
            continue;
        }
        js[i]->submit_s -= t0;
        js[i]->start_s -= t0;
        js[i]->end_s -= t0;
        try {
            p3g::fill_result(*js[i], &results[i]);
        } catch (const std::bad_alloc &) {
            results[i].status = p3g::ERR_OOM;
        }
    }
    return p3g::OK;
}

P3G_API uint64_t p3g_server_peak_admitted_bytes(const p3g_server *srv) { return srv && srv->s ? srv->s->peak_bytes() : 0; }

P3G_API uint64_t p3g_job_footprint_bytes(const p3g_pcs_params_c *pcs, const p3g_instance_c *inst, uint64_t n) {
    if (!pcs || !inst) return 0;
    std::vector<p3g::Instance> v;
    for (uint64_t i = 0; i < n; i++)
        v.push_back({inst[i].air, inst[i].trace_on_device, inst[i].height, inst[i].width, inst[i].trace, inst[i].consts,
                     inst[i].n_consts});
    p3g::PcsParams pp{pcs->log_blowup,    pcs->log_folding_arity, pcs->log_final_degree, pcs->folding_pow_bits,
                      pcs->deep_pow_bits, pcs->num_queries,       pcs->query_pow_bits};
    return p3g::job_footprint_bytes(pp, v.data(), v.size());
}
