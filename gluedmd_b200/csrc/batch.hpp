// Batched multi-walker evaluation: many walkers with the same CV / bias
// structure evaluated by one graph of two launches per step.
#pragma once

#include <cuda_runtime.h>
#include <vector>

#include "../../include/glued_b200.h"
#include "force.hpp"

namespace glued {

struct BatchTuning {
    int ra = 8;       // A atoms per warp in the coordination tile (TA = 16 * ra): 4 or 8
    int parts = 0;    // finalize CTAs per walker (0: the fewest that cover its
                      // coordination rows)
    int plain = 0;    // 1: finalize as a plain stream-ordered launch; 0: as a
                      // programmatic dependent launch of the runs kernel
    int ch = 128;     // B atoms per coordination chunk (32 * B atoms per lane): 128 or 256
};

class Batch {
public:
    Batch(const std::vector<const GluedForce*>& forces, const glued_walker_desc* walkers);
    ~Batch();
    void setStream(cudaStream_t s);
    // Times the candidate tilings on the live walkers and keeps the fastest; with
    // useCache, a batch of the same signature tuned earlier in the process reuses
    // that choice without timing.
    BatchTuning autotune(bool useCache = true);
    bool lastTuneCached() const;
    void setTuning(const BatchTuning& t);
    BatchTuning tuning() const;
    // SUM_FP32 (default): plain FP32 hill and coordination sums; SUM_FP32C:
    // two-sum compensated hill sums and blocked coordination A sums.
    void setSumPrecision(int mode);
    int sumPrecision() const;
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
