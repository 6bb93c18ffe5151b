// batch_ab.h -- independent Model_AB solves of uneven grids and contour
// lengths advanced together (see batch_ab.cu).
#pragma once

#include <vector>

#include "engine.h"
#include "grouped_pass.h"

namespace ps {

class BatchAB {
public:
    // AB solves are members 0 .. ps.size() - 1, ABC triblock solves follow
    explicit BatchAB(const std::vector<ModelABParams>& ps, const std::vector<ModelABCParams>& qs = {});
    ~BatchAB();
    int size() const { return (int)(m_.size() + t_.size()); }
    int size_ab() const { return (int)m_.size(); }
    ModelAB& model(int k);
    ModelABC& model_abc(int k);   // k counts from the first ABC member (k >= size_ab())
    void set_fields(int k, const double* wA, const double* wB, bool device_ptrs);
    void set_fields_abc(int k, const double* const w[3], bool device_ptrs);
    void update(int n);
    // update() between CUDA events on the batch stream; returns the device ms
    double update_timed(int n);
    void sync();
    int launches_per_iteration() const { return launches_; }
    int launches_per_propagate() const { return launches_prop_; }
    // sum over solves of 2 Ns M: gridpoint contour steps of one iteration
    double gridpoint_steps_per_iteration() const;

private:
    struct Group {
        int naxes = 0, Ns_max = 0;
        int path[3] = {0, 0, 0};              // schedule of each axis role (in, mid, out)
        std::vector<int> members;            // solve indices, Ns descending
        std::vector<int> Ns;                  // Ns of members, same order
        GroupSolve* dev = nullptr;            // descriptors on the device
        int* prefix_dev[9] = {};              // CTA offsets per pass kind
        std::vector<int> prefix[9];
        size_t smem[9] = {};
    };
    // solves of one shape with a generic persistent sweep, in one cooperative
    // launch: n descriptors on the device, per CTAs a solve, n x 32 barrier words
    struct SweepChunk {
        int Lx = 0, Ly = 0, Lz = 0, per = 0, n = 0;
        SweepArgs* dev = nullptr;
        unsigned* bar = nullptr;
    };
    void build_group(Group& g);
    GroupSolve describe(int k) const;   // grouped-pass descriptor of member k
    PairChain* chain_of(int k) const;
    int Ns_of(int k) const;
    void build_sweeps(const std::vector<int>& members);
    void release();
    void enqueue_iteration();
    std::vector<ModelAB*> m_;
    std::vector<ModelABC*> t_;
    std::vector<Group> groups_;
    std::vector<SweepChunk> chunks_;
    std::vector<int> own_;                   // solves propagated by their own 64^3 sweep (AB and ABC indices)
    cudaStream_t st_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    int launches_ = 0, launches_prop_ = 0;
};

}  // namespace ps
