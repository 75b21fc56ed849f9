// Batched and served VBSCF work on one GPU: a pool of host workers, each with its own context
// (own stream, own memory pool), sharing the device so that the latency-bound steps of one
// solve (small kernels, host round trips of the structure solve) overlap with other solves'
// kernels.
//
//  * Batched form: many active-space instances, each with its own plan (topology resident on
//    the device for the whole run), statically balanced over the workers by estimated cost;
//    one evaluate call runs energy + gradient for every instance and returns when all are done.
//  * Serving: VBSCF solve requests (vb_scf_input) enter a FIFO queue as they arrive; a worker
//    takes the head request when the HBM budget admits its estimated footprint, solves it
//    (plan, integrals and orbitals device-resident for the solve), and posts the result with
//    its admission and completion times; polling returns completed requests.
// The reference has no counterpart (one instance per process, src/cli/run.cpp); the request
// interface mirrors its solve entry point (xmvb::cuda::solve_scf, src/cuda/vb/scf.hpp:41-46).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

using vbcore::set_error;

namespace {

using Clock = std::chrono::steady_clock;

struct Instance {
    int worker = 0;
    int n = 0;
    vb_hs_plan* plan = nullptr;
    int n_str = 0;
    double cost = 0.0;
    // host copies of the topology (the plan keeps device copies)
    std::vector<uint64_t> alpha, beta;
    std::vector<int32_t> det_a, det_b, term_str;
    std::vector<int64_t> term_off;
    std::vector<double> term_coef;
};

struct ScfRequest {
    int64_t tag = 0;
    size_t bytes = 0;
    vb_scf_input in{};
    vb_scf_options opt{};
    std::vector<double> charges, coords, exps, coefs, c0;
    std::vector<int32_t> shell_atom, shell_nprim, orb_off, orb_fun;
    std::string structures;
    Clock::time_point submitted;
    // point the input block at this object's own copies (after every move)
    void bind() {
        in.charges = charges.data();
        in.coords = coords.data();
        in.shell_atom = shell_atom.data();
        in.shell_nprim = shell_nprim.data();
        in.shell_exponents = exps.data();
        in.shell_coefficients = coefs.data();
        in.orbital_offsets = orb_off.data();
        in.orbital_functions = orb_fun.data();
        in.structures = structures.c_str();
    }
};

struct ScfDone {
    int64_t tag;
    double energy, gradient_inf, wait_s, total_s;
    int iterations, converged;
    vb_status status;
};

size_t binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return (size_t)(r + 0.5);
}

// Device footprint estimate of one VBSCF solve (spin-pair records at full rank, determinant
// band, eigensolver workspace), used for admission.
size_t scf_bytes(int n_act, int n_el, int mult) {
    const int ka = (n_el + mult - 1) / 2, kb = n_el - ka;
    const size_t Na = binom(n_act, ka), Nb = binom(n_act, kb);
    const size_t np = (size_t)n_act * (n_act + 1) / 2;
    const size_t rec = (Na * (Na + 1) / 2 + (ka == kb ? 0 : Nb * (Nb + 1) / 2)) * (np + 6) * 8;
    const size_t ndet = std::min(Na * Nb, (size_t)4000000);
    const size_t band = std::min<size_t>((size_t)1 << 30, ndet * ndet * 16);
    const size_t nstr = std::max<size_t>(1, ndet / 4);
    return rec + band + 8 * nstr * nstr * 8 + ((size_t)64 << 20);
}

}  // namespace

struct vb_engine {
    int device = 0;
    size_t budget = 0;
    std::vector<vb_context*> ctx;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    bool stop = false;
    // batched form
    std::vector<Instance> instances;
    std::vector<std::vector<std::function<void()>>> batch_tasks;  // per worker
    int batch_pending = 0;
    // serving
    std::deque<ScfRequest> queue;
    size_t in_use = 0;
    int running = 0;
    std::vector<ScfDone> done;
    std::string error;

    void worker_loop(int w) {
        cudaSetDevice(device);
        for (;;) {
            std::unique_lock<std::mutex> lock(mu);
            cv.wait(lock, [&] {
                return stop || !batch_tasks[w].empty() ||
                       (!queue.empty() && (in_use + queue.front().bytes <= budget || running == 0));
            });
            if (stop) return;
            if (!batch_tasks[w].empty()) {
                auto tasks = std::move(batch_tasks[w]);
                batch_tasks[w].clear();
                lock.unlock();
                for (auto& t : tasks) t();
                lock.lock();
                batch_pending -= 1;
                done_cv.notify_all();
                continue;
            }
            ScfRequest req = std::move(queue.front());
            queue.pop_front();
            in_use += req.bytes;
            ++running;
            lock.unlock();
            cv.notify_all();
            ScfDone d{};
            d.tag = req.tag;
            const auto t_admit = Clock::now();
            d.wait_s = std::chrono::duration<double>(t_admit - req.submitted).count();
            vb_scf_problem* prob = nullptr;
            req.bind();
            d.status = vb_scf_problem_create(ctx[w], &req.in, &prob);
            if (d.status == VB_OK) {
                vb_scf_result res{};
                d.status = vb_solve_scf(prob, req.c0.data(), &req.opt, &res, nullptr);
                d.energy = res.energy;
                d.gradient_inf = res.gradient_inf;
                d.iterations = res.iterations;
                d.converged = res.converged;
            }
            if (prob) vb_scf_problem_destroy(prob);
            d.total_s = std::chrono::duration<double>(Clock::now() - req.submitted).count();
            lock.lock();
            if (d.status != VB_OK && error.empty()) error = vb_last_error(ctx[w]);
            in_use -= req.bytes;
            --running;
            done.push_back(d);
            lock.unlock();
            cv.notify_all();
            done_cv.notify_all();
        }
    }
};

extern "C" {

vb_status vb_engine_create(int device, size_t hbm_budget_bytes, int n_workers, vb_engine** out) {
    if (!out || n_workers < 1) return set_error(nullptr, VB_ERR_INVALID, "vb_engine_create: bad arguments");
    *out = nullptr;
    auto e = new vb_engine();
    e->device = device;
    for (int w = 0; w < n_workers; ++w) {
        vb_context* c = nullptr;
        vb_status st = vb_context_create(device, hbm_budget_bytes, &c);
        if (st != VB_OK) {
            for (auto* x : e->ctx) vb_context_destroy(x);
            delete e;
            return st;
        }
        e->ctx.push_back(c);
    }
    e->budget = e->ctx[0]->budget;
    e->batch_tasks.resize(n_workers);
    for (int w = 0; w < n_workers; ++w) e->threads.emplace_back([e, w] { e->worker_loop(w); });
    *out = e;
    return VB_OK;
}

vb_status vb_engine_destroy(vb_engine* e) {
    if (!e) return VB_OK;
    {
        std::lock_guard<std::mutex> lock(e->mu);
        e->stop = true;
    }
    e->cv.notify_all();
    for (auto& t : e->threads) t.join();
    for (auto& inst : e->instances)
        if (inst.plan) vb_hs_plan_destroy(inst.plan);
    for (auto* c : e->ctx) vb_context_destroy(c);
    delete e;
    return VB_OK;
}

const char* vb_engine_last_error(const vb_engine* e) { return e ? e->error.c_str() : ""; }

vb_status vb_engine_add_instance(vb_engine* e, const vb_expansion* ex, int64_t* id) {
    if (!e || !ex || !id) return VB_ERR_INVALID;
    Instance inst;
    inst.n = ex->n_orbitals;
    inst.alpha.assign(ex->alpha_strings, ex->alpha_strings + ex->n_alpha_strings);
    inst.beta.assign(ex->beta_strings, ex->beta_strings + ex->n_beta_strings);
    inst.det_a.assign(ex->det_alpha, ex->det_alpha + ex->n_determinants);
    inst.det_b.assign(ex->det_beta, ex->det_beta + ex->n_determinants);
    inst.term_off.assign(ex->term_offsets, ex->term_offsets + ex->n_determinants + 1);
    const int64_t nt = ex->term_offsets[ex->n_determinants];
    inst.term_str.assign(ex->term_structure, ex->term_structure + nt);
    inst.term_coef.assign(ex->term_coefficient, ex->term_coefficient + nt);
    inst.n_str = ex->n_structures;
    // cost model: determinant pairs plus the structure solve
    inst.cost = (double)ex->n_determinants * ex->n_determinants + 50.0 * (double)inst.n_str * inst.n_str;
    // least-loaded worker by accumulated cost
    std::vector<double> load(e->ctx.size(), 0.0);
    for (auto& o : e->instances) load[o.worker] += o.cost;
    inst.worker = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    vb_expansion x = *ex;
    x.alpha_strings = inst.alpha.data();
    x.beta_strings = inst.beta.data();
    x.det_alpha = inst.det_a.data();
    x.det_beta = inst.det_b.data();
    x.term_offsets = inst.term_off.data();
    x.term_structure = inst.term_str.data();
    x.term_coefficient = inst.term_coef.data();
    vb_status st = vb_hs_plan_create(e->ctx[inst.worker], &x, &inst.plan);
    if (st != VB_OK) {
        e->error = vb_last_error(e->ctx[inst.worker]);
        return st;
    }
    *id = (int64_t)e->instances.size();
    e->instances.push_back(std::move(inst));
    return VB_OK;
}

// Energy (lowest structure root) and gradient with respect to S, h and the RI factors of every
// listed instance (host buffers; ri_factors[i] is np x n_aux[i], column-major).
vb_status vb_engine_evaluate_instances(vb_engine* e, int count, const int64_t* ids, const double* const* S,
                                       const double* const* h, const double* const* eri,
                                       const double* const* ri_factors, const int* n_aux, double* energies,
                                       double* const* dS, double* const* dh, double* const* dri) {
    if (!e || count < 0 || (count > 0 && (!ids || !S || !h || !eri || !energies))) return VB_ERR_INVALID;
    std::vector<vb_status> status(count, VB_OK);
    std::vector<std::string> msg(count);
    {
        std::lock_guard<std::mutex> lock(e->mu);
        std::vector<std::vector<std::function<void()>>> per(e->ctx.size());
        for (int i = 0; i < count; ++i) {
            if (ids[i] < 0 || ids[i] >= (int64_t)e->instances.size()) return VB_ERR_INVALID;
            Instance* inst = &e->instances[ids[i]];
            per[inst->worker].push_back([=, &status, &msg] {
                vb_context* c = e->ctx[inst->worker];
                // structure H/S stay on the device (the plan's buffers); only the root returns
                const bool grad = dS && dh && dS[i] && dh[i];
                const bool ri = grad && ri_factors && ri_factors[i] && dri && dri[i];
                vb_status st = vb_hs_plan_root_gradient(inst->plan, S[i], h[i], eri[i], 1.0e-11, &energies[i], nullptr,
                                                        grad ? dS[i] : nullptr, grad ? dh[i] : nullptr,
                                                        ri ? ri_factors[i] : nullptr, ri ? n_aux[i] : 0,
                                                        ri ? dri[i] : nullptr);
                status[i] = st;
                if (st != VB_OK) msg[i] = vb_last_error(c);
            });
        }
        for (size_t w = 0; w < per.size(); ++w) {
            if (per[w].empty()) continue;
            e->batch_tasks[w] = std::move(per[w]);
            ++e->batch_pending;
        }
    }
    e->cv.notify_all();
    {
        std::unique_lock<std::mutex> lock(e->mu);
        e->done_cv.wait(lock, [&] { return e->batch_pending == 0; });
    }
    for (int i = 0; i < count; ++i)
        if (status[i] != VB_OK) {
            e->error = "instance " + std::to_string(ids[i]) + ": " + msg[i];
            return status[i];
        }
    return VB_OK;
}

vb_status vb_engine_submit_scf(vb_engine* e, const vb_scf_input* in, const double* initial_coefficients,
                               const vb_scf_options* opt, int64_t tag) {
    if (!e || !in || !initial_coefficients || !opt) return VB_ERR_INVALID;
    ScfRequest r;
    r.tag = tag;
    r.submitted = Clock::now();
    r.opt = *opt;
    r.charges.assign(in->charges, in->charges + in->n_atoms);
    r.coords.assign(in->coords, in->coords + 3 * in->n_atoms);
    r.shell_atom.assign(in->shell_atom, in->shell_atom + in->n_shells);
    r.shell_nprim.assign(in->shell_nprim, in->shell_nprim + in->n_shells);
    int nprim = 0;
    for (int s = 0; s < in->n_shells; ++s) nprim += in->shell_nprim[s];
    r.exps.assign(in->shell_exponents, in->shell_exponents + nprim);
    r.coefs.assign(in->shell_coefficients, in->shell_coefficients + nprim);
    r.orb_off.assign(in->orbital_offsets, in->orbital_offsets + in->n_active + 1);
    r.orb_fun.assign(in->orbital_functions, in->orbital_functions + in->orbital_offsets[in->n_active]);
    r.structures = in->structures;
    r.c0.assign(initial_coefficients, initial_coefficients + (size_t)in->n_shells * in->n_active);
    r.in = *in;
    r.bytes = scf_bytes(in->n_active, in->n_electrons, in->multiplicity);
    {
        std::lock_guard<std::mutex> lock(e->mu);
        e->queue.push_back(std::move(r));
    }
    e->cv.notify_all();
    return VB_OK;
}

// Completed requests (up to `capacity`): tag, energy, gradient infinity norm, iterations,
// converged flag, status, queue wait and total latency (seconds from submission).
vb_status vb_engine_poll(vb_engine* e, int capacity, int wait, int64_t* tags, double* energies, double* gradient_inf,
                         int32_t* iterations, int32_t* converged, int32_t* status, double* wait_s, double* latency_s,
                         int* n_out) {
    if (!e || !n_out || capacity < 0) return VB_ERR_INVALID;
    std::unique_lock<std::mutex> lock(e->mu);
    if (wait) e->done_cv.wait(lock, [&] { return !e->done.empty() || (e->queue.empty() && e->running == 0); });
    const int n = std::min<int>(capacity, (int)e->done.size());
    for (int i = 0; i < n; ++i) {
        const ScfDone& d = e->done[i];
        if (tags) tags[i] = d.tag;
        if (energies) energies[i] = d.energy;
        if (gradient_inf) gradient_inf[i] = d.gradient_inf;
        if (iterations) iterations[i] = d.iterations;
        if (converged) converged[i] = d.converged;
        if (status) status[i] = d.status;
        if (wait_s) wait_s[i] = d.wait_s;
        if (latency_s) latency_s[i] = d.total_s;
    }
    e->done.erase(e->done.begin(), e->done.begin() + n);
    *n_out = n;
    return VB_OK;
}

vb_status vb_engine_pending(vb_engine* e, int* queued, int* running, size_t* bytes_in_use) {
    if (!e) return VB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(e->mu);
    if (queued) *queued = (int)e->queue.size();
    if (running) *running = e->running;
    if (bytes_in_use) *bytes_in_use = e->in_use;
    return VB_OK;
}

}  // extern "C"
