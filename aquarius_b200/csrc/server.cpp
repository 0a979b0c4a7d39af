// Serving loop: continuous batching of CCSD solves on one device.
//
// * Admission (one host thread): takes requests in arrival order once their planned
//   device bytes (ccsd_plan_query) fit in the budget beside the active solves and a slot
//   is free, reserves the bytes and the slot, and starts a worker for the request.
// * Workers (one host thread per active solve): build the request's H and solver on a
//   context with its own stream, then run its iterations back to back: each iteration is
//   queued on the stream with the copy of its energy / residual to the host, the worker
//   sleeps on the iteration's completion event (blocking sync, no spinning), checks
//   convergence, and queues the next one.  The GPU interleaves the iterations of all
//   active solves through their streams; the host work of planning and launching runs on
//   as many threads as there are active solves.  A finished solve frees its context,
//   which returns its bytes for the next admission.
// Solves share nothing on the device but the memory pool; each one runs the same kernels
// and reductions it would run alone, so its result does not depend on the mix.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
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
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_admit.notify_all();
        if (admit_thread.joinable()) admit_thread.join();
        // workers leave after their current iteration
        for (auto& w : workers)
            if (w.t.joinable()) w.t.join();
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
    std::condition_variable cv_admit, cv_done;
    std::deque<std::shared_ptr<Request>> queue;
    std::deque<ccsd_server_result> results;
    int64_t next_id = 1, submitted = 0, finished = 0;
    int64_t used_bytes = 0, peak_bytes = 0;
    int n_active = 0, peak_active = 0;
    bool stop = false;
    std::thread admit_thread;
    struct Worker {
        std::thread t;
        std::shared_ptr<std::atomic<bool>> done;
    };
    std::vector<Worker> workers;   // touched by the admission thread and the destructor only

    bool stopping() {
        std::lock_guard<std::mutex> lk(mu);
        return stop;
    }

    void plan(Request& r) {
        ccsd_options o = opts.solve;
        double fl = 0;
        int64_t by = 0;
        const int st = ccsd_plan_query(r.nirrep, r.vrt.data(), r.occ.data(), &o, opts.pack_vvvv, &fl, &by);
        if (st != CCSD_OK) throw Error(st, ccsd_last_error(nullptr));
        r.bytes = by;
        r.flops = fl;
    }

    void finish(const Request& r, int status, int iters, double e, double mp2, double conv, double t_admit,
                int64_t peak = 0, const std::string& msg = std::string(), double t_built = 0) {
        ccsd_server_result res;
        std::memset(&res, 0, sizeof(res));
        res.peak_bytes = peak;
        res.t_built = t_built;
        std::snprintf(res.message, sizeof(res.message), "%s", msg.c_str());
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
            const double t_admit = now();
            // join the workers that have finished, then start this request's
            for (auto& w : workers)
                if (w.done->load() && w.t.joinable()) w.t.join();
            workers.erase(std::remove_if(workers.begin(), workers.end(), [](Worker& w) { return !w.t.joinable(); }),
                          workers.end());
            auto done = std::make_shared<std::atomic<bool>>(false);
            workers.push_back({std::thread([this, r, t_admit, done] {
                                   run_solve(r, t_admit);
                                   done->store(true);
                               }),
                               done});
        }
    }

    void drop_front(const Request& r, int status) {
        {
            std::lock_guard<std::mutex> lk(mu);
            queue.pop_front();
        }
        finish(r, status, 0, 0, 0, 0, now());
    }

    // Stream priority of a solve: the fewer flops per iteration, the higher.  A small
    // (e.g. symmetry-blocked) solve is a chain of short dependent launches; at equal
    // priority each waits behind the long GEMM waves of the large solves sharing the GPU.
    static cudaStream_t priority_stream(double flops) {
        int least = 0, greatest = 0;
        CCSD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        double f = (std::log10(std::max(flops, 1.0)) - 10.0) / 4.0;   // 1e10 -> 0, 1e14 -> 1
        f = std::min(1.0, std::max(0.0, f));
        const int prio = greatest + (int)std::lround(f * (least - greatest));
        cudaStream_t st = nullptr;
        CCSD_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio));
        return st;
    }

    void build(Request& r, cudaStream_t stream, std::unique_ptr<Context>& ctx, std::unique_ptr<Solver>& solver) {
        ctx = std::make_unique<Context>(opts.device, stream);
        ctx->plan_threads = 2;   // several solves build at once: keep the host from oversubscription
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
        ctx->spaces = S;
        ctx->spaces_set = true;
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
        build_hamiltonian(*ctx, r.naux, r.B.data(), r.eps.data(),
                          r.nirrep > 1 && !r.aux.empty() ? r.aux.data() : nullptr, opts.pack_vvvv != 0, &H);
        std::vector<double>().swap(r.B);   // the factor is on the device now
        ccsd_options o = opts.solve;
        if (o.precision != CCSD_PREC_FP64 && !kern::split_supported()) o.precision = CCSD_PREC_FP64;
        solver = std::make_unique<Solver>(*ctx, H, o);
    }

    // one active solve, start to finish, on this worker thread
    void run_solve(std::shared_ptr<Request> r, double t_admit) {
        cudaSetDevice(opts.device);
        std::unique_ptr<Context> ctx;
        std::unique_ptr<Solver> s;
        cudaEvent_t ev = nullptr;
        cudaStream_t stream = nullptr;
        int status = CCSD_OK;
        double e = 0, c = 0, mp2 = 0;
        int it = 0;
        std::string msg;
        double t_built = 0;
        try {
            stream = priority_stream(r->flops);
            build(*r, stream, ctx, s);
            t_built = now();
            mp2 = s->mp2;
            CCSD_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming | cudaEventBlockingSync));
            while (true) {
                s->iterate_async();
                s->post_status();
                CCSD_CUDA(cudaEventRecord(ev, ctx->stream));
                CCSD_CUDA(cudaEventSynchronize(ev));
                s->check_status();
                if (s->conv < s->opts.conv_tol) break;
                if (s->iterations >= s->opts.max_iter) {
                    status = CCSD_NOT_CONVERGED;
                    break;
                }
                if (stopping()) {
                    status = CCSD_NOT_CONVERGED;
                    break;
                }
            }
            e = s->energy;
            c = s->conv;
            it = s->iterations;
        } catch (const Error& err) {
            status = err.code;
            msg = err.what();
            it = s ? s->iterations : 0;
        } catch (const std::exception& err) {
            status = CCSD_ERR_ARG;
            msg = err.what();
            it = s ? s->iterations : 0;
        }
        const int64_t peak = ctx ? ctx->peak_bytes : 0;
        if (ev) cudaEventDestroy(ev);
        try {
            s.reset();
            ctx.reset();
        } catch (...) {
        }
        if (stream) cudaStreamDestroy(stream);
        {
            std::lock_guard<std::mutex> lk(mu);
            used_bytes -= r->bytes;
            n_active--;
        }
        cv_admit.notify_all();
        finish(*r, status, it, status == CCSD_OK || status == CCSD_NOT_CONVERGED ? e : 0.0, mp2, c, t_admit, peak, msg,
               t_built);
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
