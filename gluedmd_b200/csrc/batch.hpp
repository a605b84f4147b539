// Batched multi-walker evaluation: many walkers with the same force descriptor,
// one persistent launch per step.
#pragma once

#include <cuda_runtime.h>
#include <vector>

#include "../../include/glued_b200.h"
#include "force.hpp"

namespace glued {

class Batch {
public:
    Batch(const GluedForce& f, int numWalkers, const glued_walker_desc* walkers, const double* masses);
    ~Batch();
    void setStream(cudaStream_t s);
    int autotune();
    void execute();
    void updateState(int step);
    void energies(double* out);
    void cvValues(double* out);
    int numHills();
    void setHills(const double* centers, const double* heights, int n);
    int status();

private:
    struct Impl;
    Impl* impl_;
};

}  // namespace glued
