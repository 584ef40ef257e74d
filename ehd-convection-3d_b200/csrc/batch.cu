// batch.cu -- batches of independent instances (parameter sweeps in T) on one
// GPU: one CUDA graph per step over every active instance, run to saturation
// with per-instance stopping, and the launch-shape autotuner.
//
// The reference has no counterpart (one instance per process, compile-time
// grid and launch shape, nThreads in LBM.h).  Each instance is a complete
// context (csrc/api.cu) with its own stream; a batch step is captured once per
// (active set, buffer parities, macro output) as a fork on the batch stream,
// parallel branches and a join, so that independent kernels run side by side.
// Mode 1 has one branch per instance with that instance's own step launches
// on its stream; mode 0 one branch per group of instances with the same grid
// and launch shapes, each kernel of the step one launch over the group.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "ehd.h"
#include "common.cuh"
#include "kernels.h"

using namespace ehd;

struct ehd_batch {
    int device = 0;
    int mode = 1;  // 0: grouped launches, 1: per-instance graph branches
    cudaStream_t stream = nullptr;
    std::vector<ehd_ctx *> inst;
    std::vector<char> active;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join;
    std::map<std::string, cudaGraphExec_t> graphs;
    std::map<std::string, std::vector<void *>> graph_bufs;  // descriptor arrays of a graph
};

namespace {

int err(int code, const char *msg) { return set_error(code, msg); }

int cuda_fail(const char *what, cudaError_t e) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return set_error(EHD_ERR_CUDA, m.c_str());
}

struct Dev {
    int prev = -1;
    explicit Dev(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~Dev() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

void drop(ehd_batch *b) {
    for (auto &kv : b->graphs)
        if (kv.second) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    for (auto &kv : b->graph_bufs)
        for (void *p : kv.second) cudaFree(p);
    b->graph_bufs.clear();
}

// A device copy of n host elements, recorded in bufs for release with the
// graph that uses it.
template <typename X>
int upload(const X *host, size_t n, std::vector<void *> &bufs, X **dev) {
    void *d = nullptr;
    cudaError_t e = cudaMalloc(&d, sizeof(X) * (n > 0 ? n : 1));
    if (e != cudaSuccess) return cuda_fail("batch descriptors", e);
    bufs.push_back(d);
    if ((e = cudaMemcpy(d, host, sizeof(X) * n, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail("batch descriptors", e);
    *dev = (X *)d;
    return EHD_OK;
}

// One group of instances with the same grid and launch shapes, and the
// device descriptors of its launches.
struct Group {
    int nx = 0, ny = 0, nz = 0, n = 0, bx = 0;
    size_t first = 0;  // the member whose stream carries the group's branch
    int rows = 0;  // > 0: the row kernel on this many CTAs per instance
    void *lbm = nullptr;
    ReduceDesc *red = nullptr;
    PoissonArgs pa{};
};

template <typename T, typename R>
int build_group(ehd_batch *b, const std::vector<size_t> &members, bool macros,
                std::vector<void *> &bufs, Group *g) {
    const int n = (int)members.size();
    std::vector<LbmArgs> la(n);
    std::vector<StepConst> sc(n);
    std::vector<ReduceDesc> rd(n);
    std::vector<PoissonPtrs> pp(n);
    PoissonArgs pa0{};
    for (int m = 0; m < n; ++m) {
        PoissonArgs pa{};
        int r = ctx_step_args(b->inst[members[m]], macros, &la[m], &sc[m], &rd[m], &pa);
        if (r != EHD_OK) return r;
        pp[m] = PoissonPtrs{pa.spec, pa.rowsum, pa.planesum, pa.phi00, pa.ez00,
                            pa.q, pa.qmean, pa.phip, pa.dpw};
        if (m == 0) pa0 = pa;
    }
    std::vector<unsigned char> host(lbm_group_desc_bytes<T, R>(n));
    build_lbm_group_desc<T, R>(la.data(), sc.data(), n, host.data());
    unsigned char *ld = nullptr;
    int r = upload(host.data(), host.size(), bufs, &ld);
    if (r == EHD_OK) r = upload(rd.data(), rd.size(), bufs, &g->red);
    PoissonPtrs *pd = nullptr;
    if (r == EHD_OK) r = upload(pp.data(), pp.size(), bufs, &pd);
    if (r != EHD_OK) return r;
    const ehd_params *p = ctx_params(b->inst[members[0]]);
    g->nx = p->nx;
    g->ny = p->ny;
    g->nz = p->nz;
    g->n = n;
    g->first = members[0];
    g->bx = la[0].node_bx;
    // the instances' persistent row-kernel CTAs shared among the group
    g->rows = la[0].rows_grid > 0 ? std::max(1, la[0].rows_grid / n) : 0;
    g->lbm = ld;
    g->pa = pa0;
    g->pa.grp = pd;
    g->pa.ngrp = n;
    return EHD_OK;
}

template <typename T, typename R>
int capture_groups(ehd_batch *b, const std::vector<char> &act, bool macros,
                   std::vector<void *> &bufs, cudaGraph_t *graph) {
    // instances with the same grid, domain, spacing, permittivity, voltage
    // and launch shapes form one group (the group's Poisson launches take
    // their tables and those constants from its first member)
    std::map<std::vector<double>, std::vector<size_t>> groups;
    for (size_t i = 0; i < b->inst.size(); ++i) {
        if (!act[i]) continue;
        const ehd_params *p = ctx_params(b->inst[i]);
        ehd_tuning t{};
        ctx_tuning(b->inst[i], &t);
        groups[{(double)p->nx, (double)p->ny, (double)p->nz, p->lx, p->ly, p->dz, p->eps,
                p->voltage, (double)t.lbm_kernel, (double)t.node_block_x, (double)t.fft_rows,
                (double)t.fft_cols, (double)t.poisson_path, (double)t.z_solve}]
            .push_back(i);
    }
    std::vector<Group> gl;
    for (auto &kv : groups) {
        Group g;
        int r = build_group<T, R>(b, kv.second, macros, bufs, &g);
        if (r != EHD_OK) return r;
        gl.push_back(g);
    }
    // one branch per group (on the stream of its first member), so that the
    // groups' kernels overlap: a fork on the batch stream, each group's LBM
    // half, reduction and Poisson solve in order on its branch, a join
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail("batch capture", e);
    e = cudaEventRecord(b->fork, b->stream);
    for (const Group &g : gl) {
        if (e != cudaSuccess) break;
        cudaStream_t gs = ctx_stream(b->inst[g.first]);
        e = cudaStreamWaitEvent(gs, b->fork, 0);
        if (e == cudaSuccess)
            e = g.rows > 0 ? launch_lbm_rows_group<T, R>(g.lbm, g.n, g.nx, g.ny, g.rows, macros, gs)
                           : launch_lbm_group<T, R>(g.lbm, g.n, g.nx, g.ny, g.nz, g.bx, macros, gs);
        if (e == cudaSuccess) e = launch_reduce_tables_group<R>(g.red, g.n, g.nz, gs);
        if (e == cudaSuccess) e = launch_poisson<R>(g.pa, gs);
        if (e == cudaSuccess) e = cudaEventRecord(b->join[g.first], gs);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[g.first], 0);
    }
    cudaGraph_t gr = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->stream, &gr);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        cudaGetLastError();
        return cuda_fail("batch group capture", e != cudaSuccess ? e : e2);
    }
    *graph = gr;
    return EHD_OK;
}

// the graph of one step of the active instances in their present parities
int step_graph(ehd_batch *b, const std::vector<char> &act, bool macros, cudaGraphExec_t *out) {
    // key: per instance '0' (inactive) or its parity and launch generation
    std::string key;
    for (size_t i = 0; i < b->inst.size(); ++i) {
        if (!act[i]) {
            key += '0';
            continue;
        }
        key += ctx_parity(b->inst[i]) ? '2' : '1';
        key += std::to_string(ctx_generation(b->inst[i]));
        key += ',';
    }
    key += macros ? 'm' : 'n';
    auto it = b->graphs.find(key);
    if (it != b->graphs.end()) {
        *out = it->second;
        return EHD_OK;
    }
    cudaGraph_t g = nullptr;
    if (b->mode == 0) {
        // grouped launches: one launch per kernel over each group of instances
        std::vector<void *> bufs;
        int r = EHD_OK;
        switch (ctx_precision(b->inst[0])) {
            case EHD_PREC_FP64: r = capture_groups<double, double>(b, act, macros, bufs, &g); break;
            case EHD_PREC_FP32: r = capture_groups<float, float>(b, act, macros, bufs, &g); break;
            case EHD_PREC_FP16: r = capture_groups<__half, float>(b, act, macros, bufs, &g); break;
            case EHD_PREC_BF16: r = capture_groups<__nv_bfloat16, float>(b, act, macros, bufs, &g); break;
            default: r = capture_groups<Mix16, float>(b, act, macros, bufs, &g); break;
        }
        if (r != EHD_OK) {
            for (void *p : bufs) cudaFree(p);
            return r;
        }
        cudaGraphExec_t ge = nullptr;
        cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            for (void *p : bufs) cudaFree(p);
            return cuda_fail("batch graph instantiate", e);
        }
        b->graphs[key] = ge;
        b->graph_bufs[key] = bufs;
        *out = ge;
        return EHD_OK;
    }
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail("batch capture", e);
    int r = EHD_OK;
    if ((e = cudaEventRecord(b->fork, b->stream)) != cudaSuccess) r = cuda_fail("batch fork", e);
    for (size_t i = 0; r == EHD_OK && i < b->inst.size(); ++i) {
        if (!act[i]) continue;
        ehd_ctx *c = b->inst[i];
        if ((e = cudaStreamWaitEvent(ctx_stream(c), b->fork, 0)) != cudaSuccess) {
            r = cuda_fail("batch fork wait", e);
            break;
        }
        if ((r = ctx_launch_step(c, macros)) != EHD_OK) break;
        if ((e = cudaEventRecord(b->join[i], ctx_stream(c))) != cudaSuccess ||
            (e = cudaStreamWaitEvent(b->stream, b->join[i], 0)) != cudaSuccess)
            r = cuda_fail("batch join", e);
    }
    e = cudaStreamEndCapture(b->stream, &g);
    if (r != EHD_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return r != EHD_OK ? r : cuda_fail("batch capture end", e);
    }
    cudaGraphExec_t ge = nullptr;
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail("batch graph instantiate", e);
    b->graphs[key] = ge;
    *out = ge;
    return EHD_OK;
}

// order the batch stream after (to_batch) or before (!to_batch) the
// instances' streams
int order(ehd_batch *b, const std::vector<char> &act, bool to_batch) {
    cudaError_t e = cudaSuccess;
    if (to_batch) {
        for (size_t i = 0; i < b->inst.size() && e == cudaSuccess; ++i) {
            if (!act[i]) continue;
            e = cudaEventRecord(b->join[i], ctx_stream(b->inst[i]));
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[i], 0);
        }
    } else {
        e = cudaEventRecord(b->done, b->stream);
        for (size_t i = 0; i < b->inst.size() && e == cudaSuccess; ++i)
            if (act[i]) e = cudaStreamWaitEvent(ctx_stream(b->inst[i]), b->done, 0);
    }
    return e == cudaSuccess ? EHD_OK : cuda_fail("batch stream order", e);
}

int batch_step(ehd_batch *b, const std::vector<char> &act, int nsteps) {
    int k = 0;
    bool any = false, general = false;
    for (size_t i = 0; i < b->inst.size(); ++i)
        if (act[i]) {
            any = true;
            general = general || !ctx_steady(b->inst[i]);
        }
    if (!any || nsteps <= 0) return EHD_OK;
    if (general) {
        // the first step after an upload reads the uploaded state in place:
        // every active instance takes it on its own stream
        for (size_t i = 0; i < b->inst.size(); ++i)
            if (act[i]) {
                int r = ehd_step(b->inst[i], 1);
                if (r != EHD_OK) return r;
            }
        k = 1;
    }
    if (k >= nsteps) return EHD_OK;
    int r = order(b, act, true);
    for (; r == EHD_OK && k < nsteps; ++k) {
        cudaGraphExec_t ge = nullptr;
        if ((r = step_graph(b, act, k == nsteps - 1, &ge)) != EHD_OK) break;
        cudaError_t e = cudaGraphLaunch(ge, b->stream);
        if (e != cudaSuccess) {
            r = cuda_fail("batch graph launch", e);
            break;
        }
        for (size_t i = 0; i < b->inst.size(); ++i)
            if (act[i]) ctx_commit_step(b->inst[i]);
    }
    const int r2 = order(b, act, false);
    return r != EHD_OK ? r : r2;
}

}  // namespace

int ehd_batch_create(const ehd_params *params, int n, const ehd_config *config, ehd_batch **out) {
    if (!params || !out || n < 1) return err(EHD_ERR_INVALID, "ehd_batch_create: bad arguments");
    *out = nullptr;
    ehd_config cfg{};
    if (config) cfg = *config;
    cfg.stream = nullptr;
    Dev dg(cfg.device);
    ehd_batch *b = new ehd_batch();
    b->device = cfg.device;
    auto bail = [&](int code) {
        ehd_batch_destroy(b);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(cuda_fail("batch stream", e));
    if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming)) != cudaSuccess)
        return bail(cuda_fail("batch events", e));
    for (int i = 0; i < n; ++i) {
        ehd_ctx *c = nullptr;
        int r = ehd_create(&params[i], &cfg, &c);
        if (r != EHD_OK) return bail(r);
        b->inst.push_back(c);
        b->active.push_back(1);
        cudaEvent_t ev = nullptr;
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
            return bail(cuda_fail("batch events", e));
        b->join.push_back(ev);
    }
    *out = b;
    return EHD_OK;
}

int ehd_batch_destroy(ehd_batch *b) {
    if (!b) return EHD_OK;
    Dev dg(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop(b);
    for (ehd_ctx *c : b->inst) ehd_destroy(c);
    for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return EHD_OK;
}

int ehd_batch_size(const ehd_batch *b) { return b ? (int)b->inst.size() : 0; }

int ehd_batch_set_mode(ehd_batch *b, int mode) {
    if (!b || (mode != 0 && mode != 1)) return err(EHD_ERR_INVALID, "ehd_batch_set_mode: bad arguments");
    Dev dg(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop(b);
    b->mode = mode;
    return EHD_OK;
}

int ehd_batch_instance(ehd_batch *b, int i, ehd_ctx **ctx) {
    if (!b || !ctx || i < 0 || i >= (int)b->inst.size())
        return err(EHD_ERR_INVALID, "ehd_batch_instance: bad arguments");
    *ctx = b->inst[i];
    return EHD_OK;
}

int ehd_batch_set_active(ehd_batch *b, int i, int active) {
    if (!b || i < 0 || i >= (int)b->inst.size())
        return err(EHD_ERR_INVALID, "ehd_batch_set_active: bad arguments");
    b->active[i] = active ? 1 : 0;
    return EHD_OK;
}

int ehd_batch_step(ehd_batch *b, int nsteps) {
    if (!b || nsteps < 0) return err(EHD_ERR_INVALID, "ehd_batch_step: bad arguments");
    Dev dg(b->device);
    return batch_step(b, b->active, nsteps);
}

int ehd_batch_run_to_saturation(ehd_batch *b, int sample_every, double tol, int hold,
                                int64_t max_steps, int32_t *saturated, int64_t *steps,
                                double *nu_e) {
    if (!b || sample_every < 1 || hold < 1 || !(tol > 0) || max_steps < 0)
        return err(EHD_ERR_INVALID, "ehd_batch_run_to_saturation: bad arguments");
    Dev dg(b->device);
    const size_t n = b->inst.size();
    for (size_t i = 0; i < n; ++i)
        if (b->active[i] && ctx_reference_current(b->inst[i]) == 0.0)
            return err(EHD_ERR_STATE, "ehd_batch_run_to_saturation: reference current I0 not set");
    std::vector<char> run = b->active;
    std::vector<double> prev(n, 0.0), last(n, 0.0), ia(n, 0.0);
    std::vector<int> held(n, 0), ok(n, 0), bad(n, 0);
    std::vector<char> first(n, 1);
    int64_t done = 0;
    while (done < max_steps) {
        if (std::none_of(run.begin(), run.end(), [](char a) { return a != 0; })) break;
        // as ehd_run_to_saturation: a sample is the mean of the currents after
        // the last two steps of its interval
        const int k = (int)std::min<int64_t>(sample_every, max_steps - done);
        int r = EHD_OK;
        if (k >= 2) {
            if ((r = batch_step(b, run, k - 1)) != EHD_OK) return r;
            for (size_t i = 0; i < n; ++i) {
                if (!run[i]) continue;
                ehd_diag d{};
                if ((r = ehd_diagnostics(b->inst[i], &d)) != EHD_OK) return r;
                ia[i] = d.current;
                bad[i] = d.nonfinite;
            }
        }
        if ((r = batch_step(b, run, 1)) != EHD_OK) return r;
        done += k;
        for (size_t i = 0; i < n; ++i) {
            if (!run[i]) continue;
            ehd_diag d{};
            if ((r = ehd_diagnostics(b->inst[i], &d)) != EHD_OK) return r;
            if (steps) steps[i] = done;
            if (d.nonfinite || (k >= 2 && bad[i])) {  // this instance stops; the others go on
                last[i] = d.nu_e;
                ok[i] = -1;
                run[i] = 0;
                continue;
            }
            const double nu =
                k >= 2 ? 0.5 * (ia[i] + d.current) / ctx_reference_current(b->inst[i]) : d.nu_e;
            last[i] = nu;
            if (!first[i] && std::fabs(nu - prev[i]) <= tol * std::fabs(nu)) {
                if (++held[i] >= hold) {
                    ok[i] = 1;
                    run[i] = 0;
                }
            } else {
                held[i] = 0;
            }
            prev[i] = nu;
            first[i] = 0;
        }
    }
    for (size_t i = 0; i < n; ++i) {
        if (!b->active[i]) continue;
        if (saturated) saturated[i] = ok[i];
        if (nu_e) nu_e[i] = last[i];
    }
    return EHD_OK;
}

namespace {

// average time of one batch step over `steps` steps of every instance (after
// one untimed step, which also captures a new graph if the shapes changed)
// The time of one batch step: the best of three runs of `steps` steps after a
// warm-up step (the shortest run is the one least disturbed).
int time_batch(ehd_batch *b, const std::vector<char> &act, int steps, float *ms) {
    int r = batch_step(b, act, 1);
    if (r != EHD_OK) return r;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 0.f;
    cudaError_t e = cudaSuccess;
    for (int rep = 0; rep < 3 && r == EHD_OK && e == cudaSuccess; ++rep) {
        cudaEventRecord(e0, b->stream);
        r = batch_step(b, act, steps);
        cudaEventRecord(e1, b->stream);
        e = cudaEventSynchronize(e1);
        float t = 0.f;
        if (r == EHD_OK && e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
        if (rep == 0 || t < best) best = t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r != EHD_OK) return r;
    if (e != cudaSuccess) return cuda_fail("autotune timing", e);
    *ms = best / (float)steps;
    return EHD_OK;
}

}  // namespace

// The autotuner times the whole batch, not instances alone: the instances'
// kernels share the GPU, so the shape that is fastest for a grid alone is not
// the fastest beside the others.  It runs on a scratch batch with the same
// parameters (the instances' states are left alone), one grid at a time
// (coordinate descent over the distinct grids), each knob from the best so
// far; a change is kept when it saves more than 1 % of the batch step.
int ehd_batch_autotune(ehd_batch *b, int trial_steps) {
    if (!b || trial_steps < 1) return err(EHD_ERR_INVALID, "ehd_batch_autotune: bad arguments");
    Dev dg(b->device);
    const size_t n = b->inst.size();
    std::map<std::tuple<int, int, int, double, double>, std::vector<int>> groups;
    std::vector<ehd_params> ps(n);
    for (size_t i = 0; i < n; ++i) {
        ps[i] = *ctx_params(b->inst[i]);
        groups[std::make_tuple(ps[i].nx, ps[i].ny, ps[i].nz, ps[i].lx, ps[i].ly)].push_back((int)i);
    }
    ehd_config cfg{};
    cfg.precision = ctx_precision(b->inst[0]);
    cfg.device = b->device;
    ehd_batch *s = nullptr;
    int r = ehd_batch_create(ps.data(), (int)n, &cfg, &s);
    if (r != EHD_OK) return r;
    s->mode = b->mode;
    const std::vector<char> all(n, 1);
    for (size_t i = 0; r == EHD_OK && i < n; ++i) r = ehd_initialize(s->inst[i]);
    if (r == EHD_OK) r = batch_step(s, all, 1);
    float best_ms = 0.f;
    if (r == EHD_OK) r = time_batch(s, all, trial_steps, &best_ms);
    std::vector<ehd_tuning> choice, start;
    for (auto &g : groups) {
        ehd_tuning t{};
        ehd_get_tuning(s->inst[g.second.front()], &t);
        start.push_back(t);
    }
    for (auto &g : groups) {
        if (r != EHD_OK) break;
        ehd_tuning best{};
        ehd_get_tuning(s->inst[g.second.front()], &best);
        auto apply = [&](const ehd_tuning &t) {
            for (int i : g.second)
                if (ehd_set_tuning(s->inst[i], &t) != EHD_OK) return false;
            return true;
        };
        auto trial = [&](ehd_tuning t) -> int {
            if (!apply(t)) {  // shape not allowed for this grid
                apply(best);
                return EHD_OK;
            }
            float ms = 0.f;
            int rr = time_batch(s, all, trial_steps, &ms);
            if (rr != EHD_OK) return rr;
            if (ms < 0.99f * best_ms) {
                best_ms = ms;
                best = t;
            } else {
                apply(best);
            }
            return EHD_OK;
        };
        const ehd_params &p = ps[g.second.front()];
        for (int kern = 0; r == EHD_OK && kern <= 1; ++kern)
            for (int bx = 16; r == EHD_OK && bx <= 128; bx *= 2) {
                ehd_tuning t = best;
                t.lbm_kernel = kern;
                t.node_block_x = bx;
                if (t.lbm_kernel != best.lbm_kernel || t.node_block_x != best.node_block_x) r = trial(t);
            }
        if (r == EHD_OK) {  // the split-y or the five-kernel Poisson solve
            ehd_tuning t = best;
            t.poisson_path = 1 - best.poisson_path;
            r = trial(t);
        }
        if (r == EHD_OK && !poisson_fast_size(2 * (p.nz - 1))) {  // sine transform or Thomas
            ehd_tuning t = best;
            t.z_solve = 1 - best.z_solve;
            r = trial(t);
        }
        if (!poisson_fast_size(p.nx))
            for (int rows = 1; r == EHD_OK && rows <= 32; rows *= 2) {
                ehd_tuning t = best;
                t.fft_rows = rows;
                if (rows != best.fft_rows) r = trial(t);
            }
        if (!poisson_fast_size(p.ny))
            for (int cols = 1; r == EHD_OK && cols <= 32; cols *= 2) {
                ehd_tuning t = best;
                t.fft_cols = cols;
                if (cols != best.fft_cols) r = trial(t);
            }
        choice.push_back(best);
    }
    // coordinate descent over the grids can end worse than where it began
    // (the grids' best shapes depend on one another): keep the starting
    // shapes unless the final choice beats them
    if (r == EHD_OK) {
        auto apply_all = [&](const std::vector<ehd_tuning> &ts) {
            size_t k = 0;
            for (auto &g : groups) {
                for (int i : g.second)
                    if (ehd_set_tuning(s->inst[i], &ts[k]) != EHD_OK) return false;
                ++k;
            }
            return true;
        };
        float chosen_ms = 0.f, start_ms = 0.f;
        if (apply_all(choice)) r = time_batch(s, all, trial_steps, &chosen_ms);
        if (r == EHD_OK && apply_all(start)) r = time_batch(s, all, trial_steps, &start_ms);
        if (r == EHD_OK && start_ms > 0.f && start_ms <= chosen_ms) choice = start;
    }
    ehd_batch_destroy(s);
    if (r != EHD_OK) return r;
    size_t k = 0;
    for (auto &g : groups) {
        for (int i : g.second)
            if ((r = ehd_set_tuning(b->inst[i], &choice[k])) != EHD_OK) return r;
        ++k;
    }
    drop(b);
    return EHD_OK;
}
