// batch_ab.cu -- many independent Model_AB solves, of uneven grid sizes,
// contour lengths Ns, block fractions, cells and chiN, advanced together
// (with, optionally, linear ABC triblock solves of model_abc.cu, which take
// the same paths: shared generic sweeps on 32^3 / 48^3 / 64^3 grids, grouped
// line passes on the others).
//
// The reference runs independent solves one per host thread
// (scft/polystring_AB_backThread.cc); on one B200 a single small solve
// leaves most SMs idle between launches.  Here every member keeps its own
// Model_AB state (histories, fields, Anderson ring, per-solve reductions) but
// its propagator passes run in grouped launches: one launch per line pass of
// contour step t covers every solve that still has a step t (solves sorted by
// Ns, so the active ones are a prefix), each CTA running the pass body of its
// own solve (grouped_pass.cu).  Members are grouped by the number of grid
// axes longer than one (2 or 3), which fixes the pass sequence of a step.
// Solves on grids with a persistent sweep take it instead: 32^3 and 48^3
// solves of one shape share one cooperative launch for all their contour
// steps (sweep.cu, a descriptor per solve, the CTAs split between solves),
// 64^3 solves run their own 64^3 sweep (sweep64.cu), which fills the GPU
// alone (and so do 64^3 triblocks).  One batch iteration -- all propagators,
// then every member's Q, densities and field update -- is captured once as a
// CUDA graph and replayed.
#include "batch_ab.h"

#include <algorithm>
#include <array>
#include <map>
#include <numeric>

namespace ps {

namespace {

// pass kinds of a step: (mode, axis role, second-half-step field)
const int kPass[9][3] = {{MODE_FIRST_RQM4, GROUP_AX_IN, 0}, {MODE_MID_RQM4, GROUP_AX_IN, 0},
                         {MODE_END_RQM4, GROUP_AX_IN, 0},   {MODE_FWD, GROUP_AX_MID, 0},
                         {MODE_FWD, GROUP_AX_MID, 1},       {MODE_INV, GROUP_AX_MID, 0},
                         {MODE_INV, GROUP_AX_MID, 1},       {MODE_OUTER, GROUP_AX_OUT, 0},
                         {MODE_OUTER, GROUP_AX_OUT, 1}};
enum { K_FIRST, K_MID, K_END, K_FWD, K_FWD3, K_INV, K_INV3, K_OUT, K_OUT3 };

}  // namespace

BatchAB::BatchAB(const std::vector<ModelABParams>& ps, const std::vector<ModelABCParams>& qs) {
    if (ps.empty() && qs.empty()) throw Error(-1, "a batch needs at least one solve");
    grouped_prepare();
    PS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    try {
        for (const ModelABParams& p : ps) {
            if (p.mde != 0) throw Error(-2, "batched solves use RQM4");
            const int sizes[3] = {p.Lx, p.Ly, p.Lz};
            for (int n : sizes)
                if (n > 1 && !grouped_size_supported(n))
                    throw Error(-2, "batched solves support axis lengths 16, 24, 32, 48, 64, 96, 128");
            m_.push_back(new ModelAB(p, true));
            if (m_.back()->chain()->plan().naxes < 2) throw Error(-2, "batched solves need 2D or 3D grids");
        }
        for (const ModelABCParams& q : qs) {
            const int sizes[3] = {q.Lx, q.Ly, q.Lz};
            for (int n : sizes)
                if (n > 1 && !grouped_size_supported(n))
                    throw Error(-2, "batched solves support axis lengths 16, 24, 32, 48, 64, 96, 128");
            t_.push_back(new ModelABC(q));
            if (t_.back()->chain()->plan().naxes < 2) throw Error(-2, "batched solves need 2D or 3D grids");
        }
        // persistent sweeps where the grid has one, grouped line passes for the rest
        std::vector<int> swept, passes;
        for (int k = 0; k < (int)m_.size(); k++) {
            if (m_[k]->persistent_sweep64()) own_.push_back(k);
            else if (m_[k]->persistent_sweep()) swept.push_back(k);
            else passes.push_back(k);
        }
        // triblocks likewise (their own 64^3 sweep, their grids' generic sweep,
        // else grouped line passes)
        for (int j = 0; j < (int)t_.size(); j++) {
            const int k = (int)m_.size() + j;
            if (t_[j]->persistent_sweep64()) own_.push_back(k);
            else (t_[j]->persistent_sweep() ? swept : passes).push_back(k);
        }
        build_sweeps(swept);
        // groups: same number of long axes (the step's pass sequence) and the
        // same schedule on each axis role (one kernel per grouped pass)
        auto key = [&](int k) {
            const AxisPlan& pl = chain_of(k)->plan();
            return std::array<int, 4>{pl.naxes, pl.ax[0].reg, pl.naxes == 3 ? pl.ax[1].reg : 0,
                                      pl.ax[pl.naxes - 1].reg};
        };
        std::vector<std::array<int, 4>> keys;
        for (int k : passes)
            if (std::find(keys.begin(), keys.end(), key(k)) == keys.end()) keys.push_back(key(k));
        for (const auto& kk : keys) {
            Group g;
            g.naxes = kk[0];
            g.path[0] = kk[1]; g.path[1] = kk[2]; g.path[2] = kk[3];
            for (int k : passes)
                if (key(k) == kk) g.members.push_back(k);
            std::stable_sort(g.members.begin(), g.members.end(),
                             [&](int a, int b) { return Ns_of(a) > Ns_of(b); });
            build_group(g);
            groups_.push_back(std::move(g));
        }
    } catch (...) {
        release();
        throw;
    }
}

void BatchAB::release() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    for (auto& g : groups_) {
        cudaFree(g.dev);
        for (auto* p : g.prefix_dev) cudaFree(p);
    }
    for (auto& c : chunks_) {
        cudaFree(c.dev);
        cudaFree(c.bar);
    }
    for (auto* m : m_) delete m;
    m_.clear();
    for (auto* m : t_) delete m;
    t_.clear();
    if (st_) cudaStreamDestroy(st_);
    st_ = nullptr;
}

BatchAB::~BatchAB() { release(); }

void BatchAB::build_sweeps(const std::vector<int>& members) {
    // shape -> solves, in member order
    std::map<std::array<int, 3>, std::vector<int>> by_shape;
    for (int k : members) {
        if (k < (int)m_.size()) {
            const ModelABParams& p = m_[k]->params();
            by_shape[{p.Lx, p.Ly, p.Lz}].push_back(k);
        } else {
            const ModelABCParams& p = t_[k - m_.size()]->params();
            by_shape[{p.Lx, p.Ly, p.Lz}].push_back(k);
        }
    }
    for (auto& kv : by_shape) {
        const int Lx = kv.first[0], Ly = kv.first[1], Lz = kv.first[2];
        const int resident = sweep_desc_prepare(Lx, Ly, Lz);
        const int tasks = sweep_tasks_per_phase(Lx, Ly, Lz);
        // A launch of n solves gives each per = resident / n CTAs (at most the
        // tasks of a phase) and lasts its longest solve's Ns steps, each step
        // sweep_rounds_per_step(per) rounds of tasks.  With the solves in
        // order of Ns, the launches are consecutive runs of that order; pick
        // the runs with the least total cost (dynamic programme over n).
        std::vector<int> ks = kv.second;
        std::stable_sort(ks.begin(), ks.end(), [&](int a, int b) { return Ns_of(a) > Ns_of(b); });
        const int nk = (int)ks.size();
        auto per_of = [&](int n) { return std::max(1, std::min(tasks, resident / n)); };
        std::vector<double> best(nk + 1, 0.0);
        std::vector<int> from(nk + 1, 0);
        for (int i = 1; i <= nk; i++) {
            best[i] = -1.0;
            for (int j = std::max(0, i - resident); j < i; j++) {
                const double c = best[j] + (double)Ns_of(ks[j]) * sweep_rounds_per_step(Lx, Ly, Lz, per_of(i - j));
                if (best[i] < 0.0 || c < best[i]) { best[i] = c; from[i] = j; }
            }
        }
        std::vector<std::pair<int, int>> runs;   // [i0, i1) in ks
        for (int i = nk; i > 0; i = from[i]) runs.push_back({from[i], i});
        std::reverse(runs.begin(), runs.end());
        for (const auto& run : runs) {
            const size_t i0 = (size_t)run.first;
            chunks_.emplace_back();
            SweepChunk& c = chunks_.back();
            c.Lx = Lx; c.Ly = Ly; c.Lz = Lz;
            c.n = run.second - run.first;
            c.per = per_of(c.n);
            PS_CUDA(cudaMalloc(&c.bar, 32 * sizeof(unsigned) * (size_t)c.n));
            std::vector<SweepArgs> d(c.n);
            for (int i = 0; i < c.n; i++) {
                const int k = ks[i0 + i];
                d[i] = k < (int)m_.size() ? m_[k]->sweep_descriptor() : t_[k - m_.size()]->sweep_descriptor();
                d[i].bar = c.bar + 32 * (size_t)i;
                d[i].twx = twiddle_table(Lx);
                d[i].twy = twiddle_table(Ly);
                d[i].twz = twiddle_table(Lz);
            }
            PS_CUDA(cudaMalloc(&c.dev, sizeof(SweepArgs) * d.size()));
            PS_CUDA(cudaMemcpy(c.dev, d.data(), sizeof(SweepArgs) * d.size(), cudaMemcpyHostToDevice));
        }
    }
}

PairChain* BatchAB::chain_of(int k) const {
    return k < (int)m_.size() ? m_[k]->chain() : t_[k - m_.size()]->chain();
}

int BatchAB::Ns_of(int k) const { return k < (int)m_.size() ? m_[k]->Ns() : t_[k - m_.size()]->Ns(); }

GroupSolve BatchAB::describe(int k) const {
    const PairChain& c = *chain_of(k);
    GroupSolve s{};
    s.naxes = c.plan().naxes;
    for (int a = 0; a < s.naxes; a++) {
        s.ax[a] = c.plan().ax[a];
        s.tw[a] = twiddle_table(s.ax[a].N);
    }
    for (int i3 = 0; i3 < 3; i3++) s.z[i3] = c.z(i3);
    s.u[0] = c.u(0); s.u[1] = c.u(1);
    s.L1 = c.L1(); s.L2 = c.L2();
    const int never = 1 << 30;
    if (k < (int)m_.size()) {
        const ModelAB& m = *m_[k];
        s.Ns = m.Ns();
        s.M = (double)m.M();
        s.hf = m.hist_f(); s.hc = m.hist_c();
        // lane f: A then B; lane c: B then A
        s.swf[0] = m.LA(); s.swf[1] = never;
        s.swc[0] = m.LB(); s.swc[1] = never;
        const int of[3] = {0, 1, 1}, oc[3] = {1, 0, 0};
        for (int i = 0; i < 3; i++) {
            s.fF[i] = m.factor(1, of[i]); s.fH[i] = m.factor(0, of[i]);
            s.cF[i] = m.factor(1, oc[i]); s.cH[i] = m.factor(0, oc[i]);
        }
    } else {
        const ModelABC& m = *t_[k - m_.size()];
        s.Ns = m.Ns();
        s.M = (double)m.M();
        s.hf = m.hist_f(); s.hc = m.hist_c();
        // lane f: A, B, C; lane c: C, B, A
        s.swf[0] = m.L(0); s.swf[1] = m.L(0) + m.L(1);
        s.swc[0] = m.L(2); s.swc[1] = m.L(2) + m.L(1);
        for (int i = 0; i < 3; i++) {
            s.fF[i] = m.factor(1, i); s.fH[i] = m.factor(0, i);
            s.cF[i] = m.factor(1, 2 - i); s.cH[i] = m.factor(0, 2 - i);
        }
    }
    return s;
}

void BatchAB::build_group(Group& g) {
    std::vector<GroupSolve> d(g.members.size());
    for (size_t i = 0; i < g.members.size(); i++) {
        d[i] = describe(g.members[i]);
        g.Ns.push_back(d[i].Ns);
        g.Ns_max = std::max(g.Ns_max, d[i].Ns);
    }
    PS_CUDA(cudaMalloc(&g.dev, sizeof(GroupSolve) * d.size()));
    PS_CUDA(cudaMemcpy(g.dev, d.data(), sizeof(GroupSolve) * d.size(), cudaMemcpyHostToDevice));
    for (int k = 0; k < 9; k++) {
        const int mode = kPass[k][0], ax = kPass[k][1], p3 = kPass[k][2];
        if (ax == GROUP_AX_MID && g.naxes < 3) continue;
        std::vector<int>& pre = g.prefix[k];
        pre.assign(d.size() + 1, 0);
        for (size_t i = 0; i < d.size(); i++) {
            pre[i + 1] = pre[i] + grouped_ctas(d[i], mode, ax, p3);
            const int a = ax == GROUP_AX_IN ? 0 : (ax == GROUP_AX_MID ? 1 : d[i].naxes - 1);
            g.smem[k] = std::max(g.smem[k], line_pass_smem_bytes(mode, d[i].ax[a]));
        }
        if (g.smem[k] > kLinePassSmemLimit) throw Error(-2, "a batched line pass tile does not fit in shared memory");
        PS_CUDA(cudaMalloc(&g.prefix_dev[k], sizeof(int) * pre.size()));
        PS_CUDA(cudaMemcpy(g.prefix_dev[k], pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice));
    }
}

void BatchAB::enqueue_iteration() {
    int launches = 0;
    for (const SweepChunk& c : chunks_) {
        PS_CUDA(cudaMemsetAsync(c.bar, 0, 32 * sizeof(unsigned) * (size_t)c.n, st_));
        sweep_launch_desc(c.dev, c.Lx, c.Ly, c.Lz, c.per, c.n, st_);
        launches++;
    }
    for (int k : own_) {
        if (k < (int)m_.size()) m_[k]->enqueue_propagate(st_);
        else t_[k - (int)m_.size()]->enqueue_propagate(st_);
        launches++;
    }
    int Ns_max = 0;
    for (auto& g : groups_) Ns_max = std::max(Ns_max, g.Ns_max);
    for (int t = 0; t < Ns_max; t++) {
        for (auto& g : groups_) {
            // members still running at step t: a prefix of the Ns-sorted list
            int na = 0;
            while (na < (int)g.Ns.size() && g.Ns[na] > t) na++;
            if (na == 0) continue;
            auto pass = [&](int k) {
                grouped_launch(kPass[k][0], kPass[k][1], kPass[k][2], g.path[kPass[k][1]], g.dev, g.prefix_dev[k], na,
                               g.prefix[k][na], g.smem[k], t, st_);
                launches++;
            };
            const bool three = g.naxes == 3;
            if (t == 0) pass(K_FIRST);
            if (three) pass(K_FWD);
            pass(K_OUT);
            if (three) pass(K_INV);
            pass(K_MID);
            if (three) pass(K_FWD3);
            pass(K_OUT3);
            if (three) pass(K_INV3);
            pass(K_END);
        }
    }
    launches_prop_ = launches;
    for (auto* m : m_) {
        m->enqueue_post(st_);
        launches += m->launches_per_iteration() - m->launches_per_propagate();
    }
    for (auto* m : t_) {
        m->enqueue_post(st_);
        launches += m->launches_post();
    }
    launches_ = launches;
}

ModelAB& BatchAB::model(int k) {
    if (k < 0 || k >= (int)m_.size()) throw Error(-1, "solve index out of range (or not an AB solve)");
    return *m_[k];
}

ModelABC& BatchAB::model_abc(int k) {
    const int j = k - (int)m_.size();
    if (j < 0 || j >= (int)t_.size()) throw Error(-1, "solve index out of range (or not an ABC solve)");
    return *t_[j];
}

void BatchAB::set_fields(int k, const double* wA, const double* wB, bool device_ptrs) {
    sync();
    model(k).set_fields(wA, wB, device_ptrs);
}

void BatchAB::set_fields_abc(int k, const double* const w[3], bool device_ptrs) {
    sync();
    model_abc(k).set_fields(w, device_ptrs);
}

void BatchAB::update(int n) {
    sync();
    for (auto* m : m_)
        if (!m->has_fields()) throw Error(-6, "fields of every solve must be set before the batch runs");
    for (auto* m : t_)
        if (!m->has_fields()) throw Error(-6, "fields of every solve must be set before the batch runs");
    if (!graph_) {
        PS_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t g = nullptr;
        try {
            enqueue_iteration();
        } catch (...) {
            cudaStreamEndCapture(st_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        PS_CUDA(cudaStreamEndCapture(st_, &g));
        cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw Error(-3, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    }
    for (int i = 0; i < n; i++) PS_CUDA(cudaGraphLaunch(graph_, st_));
    for (auto* m : m_) m->advance(n);
    for (auto* m : t_) m->count_iterations(n);
}

double BatchAB::update_timed(int n) {
    cudaEvent_t e0, e1;
    PS_CUDA(cudaEventCreate(&e0));
    PS_CUDA(cudaEventCreate(&e1));
    update(0);
    PS_CUDA(cudaEventRecord(e0, st_));
    update(n);
    PS_CUDA(cudaEventRecord(e1, st_));
    PS_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

void BatchAB::sync() { PS_CUDA(cudaStreamSynchronize(st_)); }

double BatchAB::gridpoint_steps_per_iteration() const {
    double s = 0.0;
    for (auto* m : m_) s += 2.0 * m->Ns() * (double)m->M();
    for (auto* m : t_) s += 2.0 * m->Ns() * (double)m->M();
    return s;
}

}  // namespace ps
