// autotune.cu -- tile schedules of the line passes chosen by measurement.
//
// Two choices per axis.  The FFT schedule: the shared-memory Stockham radix
// passes (any length), or the register-resident four-step (lengths 32..256,
// fft_core.cuh RegPlan) compiled for one or for two resident CTAs per SM --
// fewer registers and more warps against possible spills.  The tile height
// of the Stockham passes: T lines per CTA sets the CTA count, the shared
// memory per CTA (so the CTAs resident per SM) and the contiguous runs of the
// strided loads.  Which is fastest depends on the grid, the batch and the
// scheme.  The tile height never changes a line's arithmetic (bit-identical
// results); the schedule changes only the order of the FFT's roundings.
//
// PairChain::autotune times complete contour steps of the chain's own pass
// sequence (the enqueue() that the propagator graphs capture) on scratch
// histories with unit fields, over Stockham tiles of 512, 1024 and 2048
// elements and the register schedules, by coordinate descent over the axes
// (two sweeps), keeping the fastest.  Results are cached per (grid, scheme,
// batch, table layout) for the life of the process; PS_B200_AUTOTUNE=0 keeps
// the defaults (Stockham passes, 2048-element tiles).
#include "engine.h"
#include "field_kernels.h"

#include <cstdio>
#include <cstdlib>
#include <array>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

namespace ps {

namespace {

using TuneKey = std::tuple<int, int, int, int, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, std::array<int, 6>> g_tune_cache;   // elements per tile, then schedule, of each axis
std::string g_tune_log;

bool tuning_enabled() {
    const char* e = std::getenv("PS_B200_AUTOTUNE");
    return !(e && e[0] == '0');
}

}  // namespace

const char* tuning_log() {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return g_tune_log.c_str();
}

void tuning_note(const char* line) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_log += line;
}

void PairChain::autotune(cudaStream_t st) {
    if (plan_.naxes < 2 || scheme_ == SCHEME_ETDRK4 || !tuning_enabled()) return;
    const TuneKey key{Lx_, Ly_, Lz_, scheme_, nbatch_, batched_tables_ ? 1 : 0};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            for (int a = 0; a < plan_.naxes; a++) {
                set_tile_elems(plan_.ax[a], it->second[a]);
                plan_.ax[a].reg = it->second[3 + a];
            }
            return;
        }
    }
    const int cand[3] = {512, 1024, 2048};
    const int first_mode = (scheme_ == SCHEME_RQM4) ? MODE_END_RQM4 : MODE_END_OS2;
    auto fits = [&](int a, int elems) {
        LineGeom g = plan_.ax[a];
        set_tile_elems(g, elems);
        return line_pass_smem_bytes(a == 0 ? first_mode : MODE_OUTER, g) <= kLinePassSmemLimit;
    };

    // scratch: two histories of nst + 1 slices and unit Boltzmann factors
    const int nst = 2;
    const long M = M_;
    const long hstride = (long)(nst + 1) * M;
    DevBuf hf((size_t)hstride * nbatch_), hc((size_t)hstride * nbatch_), ef((size_t)M * nbatch_);
    launch_fill(hf.p, hstride * nbatch_, 1.0, st);
    launch_fill(hc.p, hstride * nbatch_, 1.0, st);
    launch_fill(ef.p, M * nbatch_, 1.0, st);
    LaneFactors lf{{ef.p, ef.p}, {ef.p, ef.p}, nst};
    cudaEvent_t e0, e1;
    PS_CUDA(cudaEventCreate(&e0));
    PS_CUDA(cudaEventCreate(&e1));
    auto time_plan = [&]() {
        enqueue(hf.p, hc.p, hstride, nst, lf, lf, M, st);   // warm
        float best = 1e30f;
        for (int r = 0; r < 3; r++) {
            PS_CUDA(cudaEventRecord(e0, st));
            enqueue(hf.p, hc.p, hstride, nst, lf, lf, M, st);
            PS_CUDA(cudaEventRecord(e1, st));
            PS_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            PS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) best = ms;
        }
        return best;
    };

    std::array<int, 3> choice = {2048, 2048, 2048}, sched = {0, 0, 0};
    for (int a = 0; a < plan_.naxes; a++) {
        set_tile_elems(plan_.ax[a], choice[a]);
        sched[a] = plan_.ax[a].reg;
    }
    const std::array<int, 3> sched0 = sched;
    std::string tried;   // every candidate's step time, for the log
    const float t_default = time_plan();
    float t_best = t_default;
    for (int sweep = 0; sweep < 2; sweep++) {
        for (int a = 0; a < plan_.naxes; a++) {
            // a schedule forced by PS_B200_REG_FFT is kept; only tiles are tuned then
            const char* rf = std::getenv("PS_B200_REG_FFT");
            const bool forced = rf && rf[0] >= '0' && rf[0] <= '2';
            const bool regok = reg_lines_per_cta(plan_.ax[a].N) > 0 && !forced;
            for (int r = 0; r <= (regok ? 2 : 0); r++) {
                if (!regok && r != sched[a]) continue;
                for (int c : cand) {
                    if (r > 0 && c != choice[a]) continue;          // the tile matters to Stockham only
                    if (r == sched[a] && c == choice[a]) continue;
                    if (!fits(a, c)) continue;
                    set_tile_elems(plan_.ax[a], c);
                    plan_.ax[a].reg = r;
                    const float t = time_plan();
                    char cbuf[64];
                    std::snprintf(cbuf, sizeof(cbuf), " ax%d:%s/%d=%.1f", a, r == 0 ? "st" : (r == 1 ? "rg1" : "rg2"), c,
                                  1e3 * t / nst);
                    tried += cbuf;
                    if (t < 0.97f * t_best) {
                        t_best = t;
                        choice[a] = c;
                        sched[a] = r;
                    }
                }
            }
            set_tile_elems(plan_.ax[a], choice[a]);
            plan_.ax[a].reg = sched[a];
        }
    }
    PS_CUDA(cudaEventDestroy(e0));
    PS_CUDA(cudaEventDestroy(e1));
    PS_CUDA(cudaStreamSynchronize(st));

    static const char* names[3] = {"stockham", "reg4step", "reg4step-2cta"};
    char line[320];
    std::snprintf(line, sizeof(line), "grid %dx%dx%d %s batch %d: schedule [%s %s %s] tile elements [%d %d %d], "
                  "step %.1f us (default [%s %s %s] %.1f us)\n", Lx_, Ly_, Lz_, scheme_ == SCHEME_RQM4 ? "RQM4" : "OS2",
                  nbatch_, names[sched[0]], plan_.naxes > 1 ? names[sched[1]] : "-",
                  plan_.naxes > 2 ? names[sched[2]] : "-", choice[0], plan_.naxes > 1 ? choice[1] : 0,
                  plan_.naxes > 2 ? choice[2] : 0, 1e3 * t_best / nst, names[sched0[0]],
                  plan_.naxes > 1 ? names[sched0[1]] : "-", plan_.naxes > 2 ? names[sched0[2]] : "-",
                  1e3 * t_default / nst);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_log += "  tried (axis:schedule/tile=us per step):" + tried + "\n";
    g_tune_cache[key] = {choice[0], choice[1], choice[2], sched[0], sched[1], sched[2]};
    g_tune_log += line;
}

}  // namespace ps
