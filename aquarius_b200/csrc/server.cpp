// Serving loop: continuous batching of CCSD solves on one device.
//
// Two host threads share a request queue:
// * admission: takes requests in arrival order once their planned device bytes
//   (ccsd_plan_query) fit in the budget beside the active solves and a slot is free;
//   builds each one's H and solver on a context with its own stream;
// * iteration: keeps exactly one iteration of every active solve queued on its stream,
//   polls completion events (no host synchronisation), decides convergence from the
//   energy / residual copied back with the iteration, and retires finished solves,
//   which frees their budget for the next admission.
// Solves share nothing on the device but the memory pool; each one runs the same kernels
// and reductions it would run alone, so its result does not depend on the mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "hbuild.hpp"
#include "solver.hpp"

namespace ccsd {
void set_global_error(const std::string& msg);   // capi.cpp

namespace {

struct Request {
    int64_t id = 0;
    int nirrep = 1;
    bool synthetic = false;
    int o = 0, v = 0;
    uint64_t seed = 0;
    std::vector<int> occ, vrt, aux;
    int naux = 0;
    std::vector<double> B, eps;
    double t_submit = 0;
    int64_t bytes = -1;
    double flops = 0;
};

struct Active {
    std::shared_ptr<Request> req;
    std::unique_ptr<Context> ctx;
    std::unique_ptr<Solver> solver;
    cudaEvent_t ev = nullptr;
    bool in_flight = false;
    double t_admit = 0;
};

}  // namespace

class Server {
public:
    explicit Server(const ccsd_server_options& o) : opts(o), t0(std::chrono::steady_clock::now()) {
        CCSD_CUDA(cudaSetDevice(opts.device));
        if (opts.max_active <= 0) opts.max_active = 16;
        if (opts.memory_budget <= 0) {
            size_t fr = 0, tot = 0;
            CCSD_CUDA(cudaMemGetInfo(&fr, &tot));
            opts.memory_budget = (int64_t)(0.9 * (double)fr);
        }
        admit_thread = std::thread([this] { admit_loop(); });
        iter_thread = std::thread([this] { iter_loop(); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_admit.notify_all();
        cv_iter.notify_all();
        if (admit_thread.joinable()) admit_thread.join();
        if (iter_thread.joinable()) iter_thread.join();
    }

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    int64_t submit(std::shared_ptr<Request> r) {
        std::lock_guard<std::mutex> lk(mu);
        r->id = next_id++;
        r->t_submit = now();
        queue.push_back(r);
        submitted++;
        cv_admit.notify_all();
        return r->id;
    }

    int poll(int max, ccsd_server_result* out) {
        std::lock_guard<std::mutex> lk(mu);
        int n = 0;
        while (n < max && !results.empty()) {
            out[n++] = results.front();
            results.pop_front();
        }
        return n;
    }

    bool wait(double timeout_s) {
        std::unique_lock<std::mutex> lk(mu);
        return cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return finished == submitted; });
    }

    void stats(int* q, int* a, int64_t* pb, int* pa) {
        std::lock_guard<std::mutex> lk(mu);
        if (q) *q = (int)queue.size();
        if (a) *a = n_active;
        if (pb) *pb = peak_bytes;
        if (pa) *pa = peak_active;
    }

private:
    ccsd_server_options opts;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_admit, cv_iter, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::unique_ptr<Active>> admitted;   // handed from admission to iteration
    std::deque<ccsd_server_result> results;
    int64_t next_id = 1, submitted = 0, finished = 0;
    int64_t used_bytes = 0, peak_bytes = 0;
    int n_active = 0, peak_active = 0;
    bool stop = false;
    std::thread admit_thread, iter_thread;

    void plan(Request& r) {
        ccsd_options o = opts.solve;
        double fl = 0;
        int64_t by = 0;
        const int st = ccsd_plan_query(r.nirrep, r.vrt.data(), r.occ.data(), &o, opts.pack_vvvv, &fl, &by);
        if (st != CCSD_OK) throw Error(st, ccsd_last_error(nullptr));
        r.bytes = by;
        r.flops = fl;
    }

    void finish(const Request& r, int status, int iters, double e, double mp2, double conv, double t_admit) {
        ccsd_server_result res;
        res.id = r.id;
        res.status = status;
        res.iterations = iters;
        res.energy = e;
        res.mp2 = mp2;
        res.conv = conv;
        res.t_submit = r.t_submit;
        res.t_admit = t_admit;
        res.t_done = now();
        res.device_bytes = r.bytes;
        res.flops_per_iter = r.flops;
        std::lock_guard<std::mutex> lk(mu);
        results.push_back(res);
        finished++;
        cv_done.notify_all();
    }

    void admit_loop() {
        cudaSetDevice(opts.device);
        while (true) {
            std::shared_ptr<Request> r;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_admit.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop) return;
                r = queue.front();
            }
            if (r->synthetic && r->occ.empty()) {
                r->occ.assign(r->nirrep, 0);
                r->vrt.assign(r->nirrep, 0);
                r->aux.assign(r->nirrep, 0);
                ccsd_synth_irreps(r->seed, r->nirrep, r->o, r->v, r->occ.data(), r->vrt.data(), r->aux.data());
            }
            if (r->bytes < 0) {
                try {
                    plan(*r);
                } catch (const std::exception& e) {
                    drop_front(*r, CCSD_ERR_PLAN);
                    continue;
                }
            }
            if (r->bytes > opts.memory_budget) {
                drop_front(*r, CCSD_ERR_OOM);
                continue;
            }
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_admit.wait(lk, [&] {
                    return stop || (n_active < opts.max_active && used_bytes + r->bytes <= opts.memory_budget);
                });
                if (stop) return;
                queue.pop_front();
                used_bytes += r->bytes;
                n_active++;
                peak_bytes = std::max(peak_bytes, used_bytes);
                peak_active = std::max(peak_active, n_active);
            }
            auto a = std::make_unique<Active>();
            a->req = r;
            a->t_admit = now();
            try {
                build(*a);
            } catch (const Error& e) {
                fail(std::move(a), e.code);
                continue;
            } catch (const std::exception& e) {
                fail(std::move(a), CCSD_ERR_ARG);
                continue;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                admitted.push_back(std::move(a));
            }
            cv_iter.notify_all();
        }
    }

    void drop_front(const Request& r, int status) {
        {
            std::lock_guard<std::mutex> lk(mu);
            queue.pop_front();
        }
        finish(r, status, 0, 0, 0, 0, now());
    }

    void build(Active& a) {
        Request& r = *a.req;
        a.ctx = std::make_unique<Context>(opts.device, nullptr);
        Spaces S;
        S.nirrep = r.nirrep;
        for (int sp = 0; sp < 2; sp++)
            for (int s = 0; s < 2; s++) {
                int off = 0;
                for (int h = 0; h < r.nirrep; h++) {
                    const int n = sp == VRT ? r.vrt[h] : r.occ[h];
                    S.n[sp][s][h] = n;
                    S.off[sp][s][h] = off;
                    off += n;
                }
            }
        a.ctx->spaces = S;
        a.ctx->spaces_set = true;
        if (r.synthetic) {
            int n = 0;
            for (int h = 0; h < r.nirrep; h++) n += r.occ[h] + r.vrt[h];
            r.naux = 0;
            for (int h = 0; h < r.nirrep; h++) r.naux += r.aux[h];
            r.eps.resize(n);
            r.B.resize((size_t)r.naux * n * n);
            const int st = ccsd_synth_problem(r.seed, r.nirrep, r.occ.data(), r.vrt.data(), r.aux.data(),
                                              r.eps.data(), r.B.data());
            if (st != CCSD_OK) throw Error(st, "synthetic generator failed");
        }
        ccsd_hamiltonian H;
        build_hamiltonian(*a.ctx, r.naux, r.B.data(), r.eps.data(),
                          r.nirrep > 1 && !r.aux.empty() ? r.aux.data() : nullptr, opts.pack_vvvv != 0, &H);
        std::vector<double>().swap(r.B);   // the factor is on the device now
        ccsd_options o = opts.solve;
        if (o.precision == CCSD_PREC_SPLIT && !kern::split_supported()) o.precision = CCSD_PREC_FP64;
        a.solver = std::make_unique<Solver>(*a.ctx, H, o);
        CCSD_CUDA(cudaEventCreateWithFlags(&a.ev, cudaEventDisableTiming));
    }

    void release(Active& a) {
        if (a.ev) cudaEventDestroy(a.ev);
        a.ev = nullptr;
        a.solver.reset();
        a.ctx.reset();
        {
            std::lock_guard<std::mutex> lk(mu);
            used_bytes -= a.req->bytes;
            n_active--;
        }
        cv_admit.notify_all();
    }

    void fail(std::unique_ptr<Active> a, int status) {
        const double mp2 = a->solver ? a->solver->mp2 : 0.0;
        const int it = a->solver ? a->solver->iterations : 0;
        try {
            release(*a);
        } catch (...) {
        }
        finish(*a->req, status, it, 0, mp2, 0, a->t_admit);
    }

    void iter_loop() {
        cudaSetDevice(opts.device);
        std::vector<std::unique_ptr<Active>> act;
        while (true) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (act.empty())
                    cv_iter.wait_for(lk, std::chrono::milliseconds(5), [&] { return stop || !admitted.empty(); });
                if (stop) break;
                for (auto& a : admitted) act.push_back(std::move(a));
                admitted.clear();
            }
            bool progressed = false;
            for (auto& a : act) {
                Solver& s = *a->solver;
                try {
                    if (!a->in_flight) {
                        s.iterate_async();
                        s.post_status();
                        CCSD_CUDA(cudaEventRecord(a->ev, a->ctx->stream));
                        a->in_flight = true;
                        progressed = true;
                        continue;
                    }
                    const cudaError_t q = cudaEventQuery(a->ev);
                    if (q == cudaErrorNotReady) continue;
                    CCSD_CUDA(q);
                    a->in_flight = false;
                    progressed = true;
                    s.check_status();
                    const bool conv = s.conv < s.opts.conv_tol;
                    if (conv || s.iterations >= s.opts.max_iter) {
                        const double e = s.energy, c = s.conv, mp2 = s.mp2;
                        const int it = s.iterations;
                        const double ta = a->t_admit;
                        auto req = a->req;
                        release(*a);
                        finish(*req, conv ? CCSD_OK : CCSD_NOT_CONVERGED, it, e, mp2, c, ta);
                        a.reset();
                    }
                } catch (const Error& e) {
                    fail(std::move(a), e.code);
                } catch (const std::exception& e) {
                    fail(std::move(a), CCSD_ERR_ARG);
                }
            }
            act.erase(std::remove(act.begin(), act.end(), nullptr), act.end());
            if (!progressed && !act.empty()) std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
        for (auto& a : act) {
            if (!a) continue;
            try {
                release(*a);
            } catch (...) {
            }
        }
    }
};

}  // namespace ccsd

struct ccsd_server_s {
    ccsd::Server* s = nullptr;
};

using namespace ccsd;

namespace {
// failures of server calls are reported through ccsd_last_error(NULL)
template <class F>
int server_guard(F f) {
    try {
        f();
        return CCSD_OK;
    } catch (const Error& e) {
        set_global_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_global_error(e.what());
        return CCSD_ERR_ARG;
    }
}
}  // namespace

extern "C" {

void ccsd_server_options_default(ccsd_server_options* o) {
    if (!o) return;
    o->device = 0;
    o->memory_budget = 0;
    o->max_active = 16;
    o->pack_vvvv = 1;
    options_default(&o->solve);
}

int ccsd_server_create(const ccsd_server_options* o, ccsd_server* out) {
    if (!out) return CCSD_ERR_ARG;
    *out = nullptr;
    return server_guard([&] {
        ccsd_server_options op;
        ccsd_server_options_default(&op);
        if (o) op = *o;
        if (op.solve.diis_damping != 0.0) throw Error(CCSD_ERR_UNSUPPORTED, "DIIS damping is not supported");
        auto* h = new ccsd_server_s;
        try {
            h->s = new Server(op);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int ccsd_server_submit_synthetic(ccsd_server s, int nirrep, int o, int v, uint64_t seed, int64_t* id) {
    if (!s || !s->s) return CCSD_ERR_ARG;
    return server_guard([&] {
        if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) throw Error(CCSD_ERR_ARG, "nirrep must be 1,2,4,8");
        if (o < nirrep || v < nirrep) throw Error(CCSD_ERR_ARG, "o and v must be at least nirrep");
        auto r = std::make_shared<Request>();
        r->synthetic = true;
        r->nirrep = nirrep;
        r->o = o;
        r->v = v;
        r->seed = seed;
        const int64_t i = s->s->submit(r);
        if (id) *id = i;
    });
}

int ccsd_server_submit_factor(ccsd_server s, int nirrep, const int* vrt, const int* occ, int naux, const double* B,
                              const double* eps, const int* aux_per_irrep, int64_t* id) {
    if (!s || !s->s) return CCSD_ERR_ARG;
    return server_guard([&] {
        if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) throw Error(CCSD_ERR_ARG, "nirrep must be 1,2,4,8");
        if (!vrt || !occ || !B || !eps || naux <= 0) throw Error(CCSD_ERR_ARG, "bad factor request");
        auto r = std::make_shared<Request>();
        r->nirrep = nirrep;
        r->vrt.assign(vrt, vrt + nirrep);
        r->occ.assign(occ, occ + nirrep);
        int n = 0;
        for (int h = 0; h < nirrep; h++) n += vrt[h] + occ[h];
        r->naux = naux;
        r->B.assign(B, B + (size_t)naux * n * n);
        r->eps.assign(eps, eps + n);
        if (aux_per_irrep) r->aux.assign(aux_per_irrep, aux_per_irrep + nirrep);
        const int64_t i = s->s->submit(r);
        if (id) *id = i;
    });
}

int ccsd_server_poll(ccsd_server s, int max, ccsd_server_result* out, int* n) {
    if (!s || !s->s || !n || (max > 0 && !out)) return CCSD_ERR_ARG;
    return server_guard([&] { *n = s->s->poll(max, out); });
}

int ccsd_server_wait(ccsd_server s, double timeout_s) {
    if (!s || !s->s) return CCSD_ERR_ARG;
    return server_guard([&] {
        if (!s->s->wait(timeout_s)) throw Error(CCSD_ERR_TIMEOUT, "requests still pending");
    });
}

int ccsd_server_stats(ccsd_server s, int* queued, int* active, int64_t* peak_bytes, int* peak_active) {
    if (!s || !s->s) return CCSD_ERR_ARG;
    return server_guard([&] { s->s->stats(queued, active, peak_bytes, peak_active); });
}

int ccsd_server_destroy(ccsd_server s) {
    if (!s) return CCSD_ERR_ARG;
    const int st = server_guard([&] { delete s->s; });
    delete s;
    return st;
}

}  // extern "C"
