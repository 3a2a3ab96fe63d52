// Many independent solves of uneven grid sizes and backends in one call
// (aspher_solve_many).
//
// No reference counterpart: the reference solves one problem per call.  The
// problems are grouped by operator (backend, grid size, domain size, E*);
// each group is one batched solve on one operator (solve_batch_impl /
// solve_batch_mixed: every kernel of the loop launched once for the whole
// group, one CUDA-graph loop, per-instance convergence masks).  Groups run
// concurrently, each on its own stream of a per-device pool driven by its
// own host thread (the batched solve keeps its host thread for the rare
// branches between graph launches), so small grids fill the SMs that large
// ones leave idle; the groups start in decreasing order of estimated cost
// (longest first).  Operators come from the per-process cache shared with
// the nested driver.
#include "../../include/aspher_b200.h"
#include "pcg.hpp"

#include <algorithm>
#include <cmath>
#include <exception>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

namespace asb {

std::shared_ptr<Operator> cached_operator(int kind, int Ns, double L, double E);  // nested.cu

namespace {

struct Group {
    int backend = 0, Ns = 0;
    double L = 1.0, E = 1.0;
    std::vector<int> idx;  // problem indices, in input order
    double cost = 0.0;
};

// relative cost of one solve: Ns^2 log2 Ns per apply, the free-space
// operator transforming a grid twice the size
double solve_cost(int backend, int Ns) {
    return (backend == ASPHER_BACKEND_FFT ? 2.0 : 1.0) * (double)Ns * Ns * std::log2((double)Ns);
}

// k-th stream of the per-device pool (non-blocking, created once, kept for
// the process: a group's graphs and operators are reused across calls)
cudaStream_t pool_stream(int dev, int k) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, cudaStream_t> pool;
    std::lock_guard<std::mutex> lk(mu);
    auto it = pool.find({dev, k});
    if (it != pool.end()) return it->second;
    cudaStream_t s = nullptr;
    ASB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    pool[{dev, k}] = s;
    return s;
}

void check_problem(const aspher_problem& p, int i) {
    auto fail = [&](const char* what) {
        throw Error(ASPHER_EINVAL, "aspher_solve_many: problem " + std::to_string(i) + ": " + what);
    };
    if (p.backend != ASPHER_BACKEND_FFT && p.backend != ASPHER_BACKEND_PERIODIC)
        fail("unknown backend (expected fft or periodic)");
    if (p.grid_size < 2 || p.grid_size > 16384) fail("grid_size must be in [2, 16384]");
    if (!p.g0_dev || !p.pressure_dev) fail("NULL gap or pressure buffer");
    if (((uintptr_t)p.g0_dev | (uintptr_t)p.pressure_dev) % 16)
        fail("buffers must be 16-byte aligned");
    if (!(p.p_bar > 0.0) || !std::isfinite(p.p_bar)) fail("p_bar must be positive");
    if (!(p.domain_size >= 0.0) || !(p.E_star >= 0.0) || !std::isfinite(p.domain_size) ||
        !std::isfinite(p.E_star))
        fail("domain_size and E_star must be positive (0: the default 1)");
}

}  // namespace

void solve_many(int n, const aspher_problem* pr, const aspher_many_opts& mo, aspher_result* res,
                aspher_result* res_float, cudaStream_t caller) {
    if (n < 1) throw Error(ASPHER_EINVAL, "aspher_solve_many: n must be >= 1");
    if (mo.precision < ASPHER_MANY_DOUBLE || mo.precision > ASPHER_MANY_FLOAT_THEN_DOUBLE)
        throw Error(ASPHER_EINVAL, "aspher_solve_many: unknown precision");
    if (!(mo.tol > 0.0)) throw Error(ASPHER_EINVAL, "aspher_solve_many: tol must be positive");
    const bool polish = mo.precision == ASPHER_MANY_FLOAT_THEN_DOUBLE;
    const double polish_tol = mo.polish_tol > 0.0 ? mo.polish_tol : mo.tol;
    if (polish && polish_tol > mo.tol)
        throw Error(ASPHER_EINVAL, "aspher_solve_many: polish_tol must be in (0, tol]");
    for (int i = 0; i < n; ++i) check_problem(pr[i], i);

    // group per operator
    std::map<std::tuple<int, int, double, double>, Group> by_op;
    for (int i = 0; i < n; ++i) {
        const double L = pr[i].domain_size > 0.0 ? pr[i].domain_size : 1.0;
        const double E = pr[i].E_star > 0.0 ? pr[i].E_star : 1.0;
        Group& g = by_op[std::make_tuple(pr[i].backend, pr[i].grid_size, L, E)];
        g.backend = pr[i].backend;
        g.Ns = pr[i].grid_size;
        g.L = L;
        g.E = E;
        g.idx.push_back(i);
        g.cost += solve_cost(g.backend, g.Ns);
    }
    std::vector<Group> groups;
    for (auto& kv : by_op) groups.push_back(std::move(kv.second));
    std::stable_sort(groups.begin(), groups.end(),
                     [](const Group& a, const Group& b) { return a.cost > b.cost; });

    int dev = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    // every operator and stream exists before any group starts (their set-up
    // synchronises the device)
    std::vector<std::shared_ptr<Operator>> ops;
    std::vector<cudaStream_t> streams;
    for (size_t k = 0; k < groups.size(); ++k) {
        ops.push_back(cached_operator(groups[k].backend, groups[k].Ns, groups[k].L, groups[k].E));
        streams.push_back(pool_stream(dev, (int)k));
    }
    // the groups start after the caller's earlier work (its gaps)
    cudaEvent_t ready = nullptr;
    ASB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    ASB_CUDA(cudaEventRecord(ready, caller));
    for (cudaStream_t s : streams) ASB_CUDA(cudaStreamWaitEvent(s, ready, 0));
    ASB_CUDA(cudaEventDestroy(ready));

    aspher_solve_opts o;
    aspher_solve_opts_default(&o);
    o.max_iter = mo.max_iter > 0 ? mo.max_iter : 5000;
    o.precond = mo.precond;
    o.precond_radius = mo.precond_radius > 0 ? mo.precond_radius : 2;
    o.keep_best = 0;
    o.light = 1;
    o.requested_tol = mo.tol;
    o.tol = polish ? polish_tol : mo.tol;
    const double float_tol = mo.float_tol > 0.0 ? mo.float_tol : mo.tol;

    auto run_group = [&](size_t k) {
        const Group& g = groups[k];
        const int B = (int)g.idx.size();
        std::vector<const double*> g0s(B);
        std::vector<double> pbars(B);
        std::vector<double*> outs(B);
        for (int b = 0; b < B; ++b) {
            const aspher_problem& p = pr[g.idx[b]];
            g0s[b] = p.g0_dev;
            pbars[b] = p.p_bar;
            outs[b] = p.pressure_dev;
        }
        std::vector<aspher_result> r(B), rf(B);
        if (mo.precision == ASPHER_MANY_DOUBLE) {
            aspher_solve_opts od = o;
            od.dtype = ASPHER_F64;
            solve_batch_impl<double>(*ops[k], od, B,
                                     reinterpret_cast<const void* const*>(g0s.data()),
                                     pbars.data(), nullptr, outs.data(), r.data(), streams[k]);
            rf = r;
        } else {
            solve_batch_mixed(*ops[k], o, B, g0s.data(), pbars.data(), float_tol, polish ? 1 : 0,
                              outs.data(), r.data(), rf.data(), streams[k]);
        }
        for (int b = 0; b < B; ++b) {
            res[g.idx[b]] = r[b];
            if (res_float) res_float[g.idx[b]] = rf[b];
        }
    };

    std::vector<std::exception_ptr> errs(groups.size());
    if (mo.concurrent && groups.size() > 1) {
        std::vector<std::thread> th;
        for (size_t k = 0; k < groups.size(); ++k)
            th.emplace_back([&, k]() {
                try {
                    ASB_CUDA(cudaSetDevice(dev));
                    run_group(k);
                } catch (...) {
                    errs[k] = std::current_exception();
                }
            });
        for (auto& t : th) t.join();
    } else {
        for (size_t k = 0; k < groups.size(); ++k) {
            try {
                run_group(k);
            } catch (...) {
                errs[k] = std::current_exception();
                break;
            }
        }
    }
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
    // later work on the caller's stream runs after every group
    for (cudaStream_t s : streams) {
        cudaEvent_t done = nullptr;
        ASB_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        ASB_CUDA(cudaEventRecord(done, s));
        ASB_CUDA(cudaStreamWaitEvent(caller, done, 0));
        ASB_CUDA(cudaEventDestroy(done));
    }
}

}  // namespace asb

extern "C" void aspher_many_opts_default(aspher_many_opts* o) {
    if (!o) return;
    o->precision = ASPHER_MANY_FLOAT_THEN_DOUBLE;
    o->tol = 1e-6;
    o->float_tol = 0.0;
    o->polish_tol = 0.0;
    o->max_iter = 5000;
    o->precond = ASPHER_PRECOND_STENCIL;
    o->precond_radius = 2;
    o->concurrent = 1;
}

extern "C" int aspher_solve_many(int n, const aspher_problem* problems,
                                 const aspher_many_opts* opts, aspher_result* res,
                                 aspher_result* res_float, void* stream) {
    try {
        if (!problems || !opts || !res)
            throw asb::Error(ASPHER_EINVAL, "aspher_solve_many: NULL argument");
        asb::solve_many(n, problems, *opts, res, res_float, static_cast<cudaStream_t>(stream));
        return ASPHER_OK;
    } catch (const asb::Error& e) {
        asb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        asb::set_last_error(e.what());
        return ASPHER_ECUDA;
    }
}
