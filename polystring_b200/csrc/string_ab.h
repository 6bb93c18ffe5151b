// string_ab.h -- batched string method context (string_ab.cu).
#pragma once

#include "engine.h"

namespace ps {

constexpr int kMaxImages = 64;   // images per string (spline arrays live in registers/local memory)

class StringAB {
public:
    // m images of which this context relaxes [lo, hi) (its shard; the whole
    // string when lo = 0, hi = m).  The string fields wa, wb, phiA, phiB are
    // held for all m images; histories and SCFT work arrays for the shard only.
    StringAB(const ModelABParams& p, int m, int max_iter, int lo = 0, int hi = -1);
    ~StringAB();
    // wa, wb: m x M (image-major); the first and last images are the ends
    void set_images(const double* wa, const double* wb, bool device_ptrs);
    void iterate(int n);                 // n string iterations (graph replays); whole string only
    void relax();                        // SCFT of the shard's images and their H (run_scftInString)
    void reparameterize();               // arc length, spline re-sampling, ends (all m images)
    void H(double* out);                 // free energy of every image (last iteration)
    void S(double* out);                 // normalised arc length of every image
    void get(int which, double* out, bool device_dst);   // 0 wa, 1 wb, 2 phiA, 3 phiB (m x M)
    double* device_ptr(int which);       // the same arrays in device memory
    void sync();
    int images() const { return m_; }
    int shard_lo() const { return lo_; }
    int shard_hi() const { return lo_ + nloc_; }
    long M() const { return M_; }
    int Ns() const { return Ns_; }
    int launches_per_iteration() const;
    bool cluster_sweep() const { return use_cluster_; }
    cudaStream_t stream() const { return st_; }

private:
    void enqueue_scft_iteration();
    void enqueue_relax();
    void enqueue_reparameterize();
    void enqueue_string_iteration();
    cudaGraphExec_t capture(void (StringAB::*enq)());
    ModelABParams p_;
    int m_, max_iter_;
    int lo_ = 0, nloc_ = 0;              // shard: images lo_ .. lo_ + nloc_ - 1
    long M_;
    int LA_, LB_, Ns_;
    double dsA_, dsB_;
    PairChain* chain_ = nullptr;
    cudaStream_t st_ = nullptr;
    cudaGraphExec_t giter_ = nullptr, grelax_ = nullptr, grepar_ = nullptr;
    DevBuf hf_, hc_, wa_, wb_, yita_, phiA_, phiB_, eFA_, eHA_, eFB_, eHB_, ends_, cA_, cB_, scal_, S_, partial_;
    // one thread-block cluster per image for the propagators (2D grids that have one)
    bool use_cluster_ = false;
    DevBuf clK_;                         // per-axis exp(h k^2): x, y for h = ds, then ds / 2
    long iters_ = 0;
    bool relaxed_ = false;
    bool ready_ = false;
};

}  // namespace ps
