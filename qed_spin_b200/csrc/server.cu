// =============================================================================
// server.cu -- the request server: eigs, thermal (one block's FTLM) and T = 0 dynamics solves of sectors of
// different sizes, served with continuous batching on one GPU.
//
// Requests queue in arrival order. A worker admits the head of the queue when a slot is free and the request's
// estimated HBM footprint (sectors, reduced CSRs, Krylov vectors) fits what the budget has left; a request
// larger than the whole budget runs alone. So requests that arrive while others are on the GPU are admitted as
// slots and memory free up, and each admitted request runs on its worker thread's own CUDA stream (the library
// is built with per-thread default streams): the solves' kernels overlap on the device. A worker's thread
// allowance caps the optional buffers its solve may plan with (a kept Krylov basis) to what it was admitted
// with. Every solve runs the same drivers as a direct call, so a request's result does not depend on what else
// is in flight.
// =============================================================================
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "qb_internal.cuh"

namespace qb {
namespace {

struct SectorCopy {
    qb_sector_desc d{};
    std::vector<int32_t> perms;
    std::vector<uint64_t> flips;
    std::vector<double> chars;
    void take(const qb_sector_desc& s) {
        d = s;
        if (s.n_sites < 1 || s.n_sites > 64 || s.group_size < 1 || !s.perms || !s.chars)
            throw Error(QB_EINVAL, "request: malformed sector");
        perms.assign(s.perms, s.perms + static_cast<std::size_t>(s.group_size) * s.n_sites);
        chars.assign(s.chars, s.chars + 2 * static_cast<std::size_t>(s.group_size));
        if (s.flips) flips.assign(s.flips, s.flips + s.group_size);
        d.perms = perms.data();
        d.chars = chars.data();
        d.flips = s.flips ? flips.data() : nullptr;
    }
};

struct ProgramCopy {
    qb_program_desc d{};
    std::vector<uint64_t> gflip, vval, tsign;
    std::vector<int32_t> gset;
    std::vector<uint32_t> gvb, vtb;
    std::vector<double> coeff;
    void take(const qb_program_desc& p) {
        d = p;
        if (!p.group_flip || !p.group_setbits || !p.group_vbegin || !p.vsub_val || !p.vsub_tbegin || !p.term_sign ||
            !p.term_coeff)
            throw Error(QB_EINVAL, "request: malformed program");
        gflip.assign(p.group_flip, p.group_flip + p.n_groups);
        gset.assign(p.group_setbits, p.group_setbits + p.n_groups);
        gvb.assign(p.group_vbegin, p.group_vbegin + p.n_groups + 1);
        vval.assign(p.vsub_val, p.vsub_val + p.n_vsub);
        vtb.assign(p.vsub_tbegin, p.vsub_tbegin + p.n_vsub + 1);
        tsign.assign(p.term_sign, p.term_sign + p.n_terms);
        coeff.assign(p.term_coeff, p.term_coeff + 2 * static_cast<std::size_t>(p.n_terms));
        d.group_flip = gflip.data();
        d.group_setbits = gset.data();
        d.group_vbegin = gvb.data();
        d.vsub_val = vval.data();
        d.vsub_tbegin = vtb.data();
        d.term_sign = tsign.data();
        d.term_coeff = coeff.data();
    }
};

struct Job {
    std::uint64_t ticket = 0;
    int kind = QB_REQ_EIGS;
    SectorCopy sec, tgt;
    ProgramCopy h, op;
    int k = 1, krylov = 200;
    std::vector<double> omega, betas;
    double eta = 0.05;
    int samples = 0;
    std::uint64_t seed = 0;
    std::uint64_t footprint = 0, allowance = 0, csr_budget = 0;
    double t_submit = 0.0, t_admit = -1.0, t_done = -1.0;
    bool done = false;
    int status = QB_OK;
    std::string error;
    std::vector<double> values, S;
    double e0 = 0.0, conv_change = 0.0;
    int converged = 0, matvecs = 0;
};

double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// An upper estimate of a sector's dimension before it is enumerated: C(N, n_up) / |G|, plus the excess of
// states with smaller orbits (at most a quarter at these sizes) and a floor.
std::uint64_t estimate_dim(const qb_sector_desc& d) {
    return static_cast<std::uint64_t>(1.25 * binom(d.n_sites, d.n_up) / std::max(1, d.group_size)) + 64;
}

// Device bytes: a sector (representatives, 1/norms, hash slots at load <= 1/2, tables); its reduced CSR (about
// half the program's groups act on a row, 5 bytes an entry, the row pointers); Krylov vectors of 16 bytes.
std::uint64_t sector_bytes(std::uint64_t n) { return n * (8 + 8 + 64) + (4ULL << 20); }
std::uint64_t csr_bytes(std::uint64_t n, const qb_program_desc& p) { return n * (8 + 5 * (p.n_groups / 2 + 2)); }

void plan(Job& j, std::uint64_t budget) {
    const std::uint64_t n = estimate_dim(j.sec.d);
    std::uint64_t fixed = sector_bytes(n), csr = csr_bytes(n, j.h.d), work = 0, keep = 0;
    if (j.kind == QB_REQ_THERMAL) {
        work = static_cast<std::uint64_t>(j.samples) * 16 * 4 * n + 16 * n;   // three sample blocks, w, the start
    } else if (j.kind == QB_REQ_EIGS) {
        if (j.k <= 1) {
            work = 48 * n;   // the recurrence's w and two vectors
        } else {
            const std::uint64_t p = j.k + std::max(j.k / 2, 8);
            const std::uint64_t m = std::min<std::uint64_t>(2 * p + 20, 2 * j.k + 60);
            work = (m + 2 + p + j.k) * 16 * n;
        }
    } else {
        const std::uint64_t nt = estimate_dim(j.tgt.d);
        fixed += sector_bytes(nt);
        csr += csr_bytes(nt, j.h.d);
        work = 96 * n + 64 * nt;   // ground state: seed, w, u and the recurrence; phi and the fraction's recurrence
        keep = std::min<std::uint64_t>(610 * 16 * n, budget / 8);   // a kept basis for the ground state's Ritz vector
    }
    j.csr_budget = csr;
    j.footprint = fixed + csr + work + keep;
    // what the solve may plan its optional buffers with: the kept basis it was admitted with, as the lanes'
    // half-of-available rule reads it
    j.allowance = 2 * (keep + work) + 1;
}

}  // namespace
}  // namespace qb

struct qb_server {
    int device = 0;
    int max_active = 1;
    std::uint64_t budget = 0, in_use = 0;
    int active = 0;
    bool stop = false;
    std::uint64_t next_ticket = 1;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<qb::Job>> pending;
    std::map<std::uint64_t, std::shared_ptr<qb::Job>> jobs;
    std::vector<std::thread> workers;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }

    bool admissible() const {
        if (pending.empty() || active >= max_active) return false;
        const auto& j = pending.front();
        return active == 0 || in_use + j->footprint <= budget;
    }

    void run(qb::Job& j);

    void worker() {
        cudaSetDevice(device);
        for (;;) {
            std::shared_ptr<qb::Job> j;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || admissible(); });
                if (stop) return;
                j = pending.front();
                pending.pop_front();
                in_use += j->footprint;
                ++active;
                j->t_admit = now();
            }
            qb::set_thread_allowance(j->allowance);
            run(*j);
            qb::set_thread_allowance(0);
            {
                std::lock_guard<std::mutex> lk(mu);
                in_use -= j->footprint;
                --active;
                j->t_done = now();
                j->done = true;
            }
            cv_work.notify_all();
            cv_done.notify_all();
        }
    }
};

namespace {

// Releases the library objects of one solve (sectors come from the registry: a block that recurs across
// requests is enumerated once).
struct Owned {
    std::vector<qb_sector*> secs;
    std::vector<qb_program*> progs;
    std::vector<qb_csr*> csrs;
    ~Owned() {
        for (auto* c : csrs) qb_csr_destroy(c);
        for (auto* p : progs) qb_program_destroy(p);
        for (auto* s : secs) qb_sector_release(s);
    }
};

int step(int rc, qb::Job& j) {
    if (rc != QB_OK && j.status == QB_OK) {
        j.status = rc;
        j.error = qb_last_error();
    }
    return rc;
}

}  // namespace

void qb_server::run(qb::Job& j) {
    Owned o;
    auto sector = [&](const qb_sector_desc& d) -> qb_sector* {
        qb_sector* s = nullptr;
        if (step(qb_sector_acquire(&d, &s), j) != QB_OK) return nullptr;
        o.secs.push_back(s);
        return s;
    };
    auto program = [&](const qb_program_desc& d) -> qb_program* {
        qb_program* p = nullptr;
        if (step(qb_program_create(&d, &p), j) != QB_OK) return nullptr;
        o.progs.push_back(p);
        return p;
    };
    // the reduced CSR when it fits what the request was admitted with; else the walk
    auto lane = [&](qb_sector* s, qb_program* p) {
        qb_csr* c = nullptr;
        if (qb_csr_build(s, s, p, j.csr_budget, &c) == QB_OK) {
            o.csrs.push_back(c);
            qb_program_attach_csr(p, c);
        }
    };
    if (j.kind == QB_REQ_EIGS) {
        qb_sector* s = sector(j.sec.d);
        qb_program* p = s ? program(j.h.d) : nullptr;
        if (!p) return;
        lane(s, p);
        if (j.k <= 1) {
            double e0 = 0.0;
            int it = 0, cv = 0, mv = 0;
            if (step(qb_eigs_lowest(s, p, 0, QB_C128, 0, &e0, &it, &cv, &mv), j) != QB_OK) return;
            j.values = {e0};
            j.converged = cv;
            j.matvecs = mv;
        } else {
            std::vector<double> v(j.k);
            int nf = 0, cv = 0, mv = 0;
            if (step(qb_eigs_k(s, p, j.k, 0, v.data(), &nf, &cv, &mv, nullptr), j) != QB_OK) return;
            v.resize(std::max(0, nf));
            j.values = v;
            j.converged = cv;
            j.matvecs = mv;
        }
    } else if (j.kind == QB_REQ_THERMAL) {
        qb_sector* s = sector(j.sec.d);
        qb_program* p = s ? program(j.h.d) : nullptr;
        if (!p) return;
        lane(s, p);
        const std::size_t nb = j.betas.size();
        j.S.assign(3 * nb, 0.0);
        double e_min = 0.0;
        if (step(qb_ftlm(s, p, j.samples, j.krylov, j.seed, j.betas.data(), static_cast<int>(nb), QB_C128, j.S.data(),
                         j.S.data() + nb, j.S.data() + 2 * nb, &e_min),
                 j) != QB_OK)
            return;
        j.values = {e_min};
        j.converged = 1;
    } else {
        qb_sector* src = sector(j.sec.d);
        qb_sector* tgt = src ? sector(j.tgt.d) : nullptr;
        qb_program* hs = tgt ? program(j.h.d) : nullptr;
        qb_program* ht = hs ? program(j.h.d) : nullptr;
        qb_program* op = ht ? program(j.op.d) : nullptr;
        if (!op) return;
        lane(src, hs);
        if (qb_sector_dim(tgt) > 0) lane(tgt, ht);
        j.S.assign(j.omega.size(), 0.0);
        int cert = 0;
        if (step(qb_dynamics_t0(src, hs, tgt, ht, op, j.krylov, j.omega.data(), static_cast<int>(j.omega.size()), j.eta,
                                j.S.data(), &j.e0, &j.conv_change, &cert),
                 j) != QB_OK)
            return;
        j.converged = cert;
        j.values = {j.e0};
    }
}

extern "C" {

int qb_server_create(int max_active, uint64_t hbm_budget, qb_server** out) {
    return qb::guarded([&] {
        using namespace qb;
        if (!out || max_active < 1 || max_active > 64) throw Error(QB_EINVAL, "max_active must be in [1, 64]");
        auto s = std::make_unique<qb_server>();
        cuda_check(cudaGetDevice(&s->device), "device");
        s->max_active = max_active;
        if (hbm_budget == 0) {
            std::size_t free_b = 0, total_b = 0;
            cuda_check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
            hbm_budget = static_cast<uint64_t>(0.8 * static_cast<double>(free_b));
        }
        s->budget = hbm_budget;
        for (int i = 0; i < max_active; ++i) s->workers.emplace_back([p = s.get()] { p->worker(); });
        *out = s.release();
    });
}

int qb_server_submit(qb_server* s, const qb_request* r, uint64_t* ticket) {
    return qb::guarded([&] {
        using namespace qb;
        if (!s || !r || !ticket) throw Error(QB_EINVAL, "null argument");
        if (r->kind != QB_REQ_EIGS && r->kind != QB_REQ_DYNAMICS && r->kind != QB_REQ_THERMAL)
            throw Error(QB_EINVAL, "request: unknown kind");
        auto j = std::make_shared<Job>();
        j->kind = r->kind;
        j->sec.take(r->sector);
        j->h.take(r->h);
        j->k = r->k;
        if (r->kind == QB_REQ_EIGS && (r->k < 1 || r->k > QB_SERVER_MAX_LEVELS))
            throw Error(QB_EINVAL, "request: k must be in [1, 16]");
        if (r->kind == QB_REQ_THERMAL) {
            if (r->samples < 1 || r->samples > 64) throw Error(QB_EINVAL, "request: samples must be in [1, 64]");
            if (r->krylov < 2) throw Error(QB_EINVAL, "request: krylov must be >= 2");
            if (!r->betas || r->n_beta < 1) throw Error(QB_EINVAL, "request: no temperatures");
            j->samples = r->samples;
            j->krylov = r->krylov;
            j->seed = r->seed;
            j->betas.assign(r->betas, r->betas + r->n_beta);
        }
        if (r->kind == QB_REQ_DYNAMICS) {
            j->tgt.take(r->target);
            j->op.take(r->op);
            if (r->target.n_sites != r->sector.n_sites) throw Error(QB_EINVAL, "request: sectors of different sizes");
            if (!r->omega || r->n_omega < 1) throw Error(QB_EINVAL, "request: no frequencies");
            j->omega.assign(r->omega, r->omega + r->n_omega);
            j->krylov = r->krylov;
            j->eta = r->eta;
        }
        plan(*j, s->budget);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->stop) throw Error(QB_EINVAL, "server is closing");
            j->ticket = s->next_ticket++;
            j->t_submit = s->now();
            s->jobs[j->ticket] = j;
            s->pending.push_back(j);
        }
        s->cv_work.notify_all();
        *ticket = j->ticket;
    });
}

int qb_server_wait(qb_server* s, uint64_t ticket, int timeout_ms, qb_result* out, double* S) {
    if (!s || !out) {
        qb::set_last_error("null argument");
        return QB_EINVAL;
    }
    std::shared_ptr<qb::Job> j;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->jobs.find(ticket);
        if (it == s->jobs.end()) {
            qb::set_last_error("unknown ticket");
            return QB_EINVAL;
        }
        j = it->second;
        const auto ready = [&] { return j->done; };
        if (timeout_ms < 0)
            s->cv_done.wait(lk, ready);
        else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
            qb::set_last_error("not done");
            return QB_ETIMEOUT;
        }
        s->jobs.erase(it);
    }
    std::memset(out, 0, sizeof(*out));
    out->status = j->status;
    out->n_values = static_cast<int>(std::min<std::size_t>(j->values.size(), QB_SERVER_MAX_LEVELS));
    for (int i = 0; i < out->n_values; ++i) out->values[i] = j->values[i];
    out->converged = j->converged;
    out->matvecs = j->matvecs;
    out->e0 = j->e0;
    out->conv_change = j->conv_change;
    out->t_submit = j->t_submit;
    out->t_admit = j->t_admit;
    out->t_done = j->t_done;
    out->footprint = j->footprint;
    if (S && !j->S.empty()) std::copy(j->S.begin(), j->S.end(), S);
    if (j->status != QB_OK) qb::set_last_error(j->error);
    return QB_OK;
}

int qb_server_clock(qb_server* s, double* seconds) {
    if (!s || !seconds) return QB_EINVAL;
    *seconds = s->now();
    return QB_OK;
}

int qb_server_destroy(qb_server* s) {
    return qb::guarded([&] {
        if (!s) return;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;   // requests still queued are dropped; admitted ones finish
        }
        s->cv_work.notify_all();
        for (auto& t : s->workers) t.join();
        delete s;
    });
}

}  // extern "C"
