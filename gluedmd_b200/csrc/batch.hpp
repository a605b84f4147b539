// Batched multi-walker evaluation: many walkers with the same CV / bias
// structure evaluated by one graph of two launches per step.
#pragma once

#include <cuda_runtime.h>
#include <vector>

#include "../../include/glued_b200.h"
#include "force.hpp"

namespace glued {

struct BatchTuning {
    int ra = 8;       // A atoms per thread in the coordination tile (TA = 16 * ra)
    int parts = 0;    // finalize CTAs per walker (0: the fewest that cover its
                      // coordination rows)
    int plain = 0;    // 1: finalize as a plain stream-ordered launch; 0: as a
                      // programmatic dependent launch of the runs kernel
};

class Batch {
public:
    Batch(const std::vector<const GluedForce*>& forces, const glued_walker_desc* walkers);
    ~Batch();
    void setStream(cudaStream_t s);
    BatchTuning autotune();
    void setTuning(const BatchTuning& t);
    BatchTuning tuning() const;
    void execute();
    void updateState(int step);
    void energies(double* out);
    void cvValues(double* out);
    int numCVs() const;
    int numWalkers() const;
    int numHills();
    void setHills(const double* centers, const double* heights, int n);
    void getHills(double* centers, double* heights, int n);
    int status();
    long long launchCount() const;
    bool graphed() const;
    double lastStepMs();
    void phaseTimes(double* out);
    long long phaseStamps(unsigned long long* out, long long cap);

private:
    struct Impl;
    Impl* impl_;
};

}  // namespace glued
