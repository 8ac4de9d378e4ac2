// Liquid-volume transport (liquid.cu): device-resident state and one
// interval's inputs, shared by the standalone state (rb200_liquid_*) and the
// carrier's liquid step (carrier.cu).
#pragma once

#include "internal.hpp"

namespace rb200 {

// One interval's inputs (src/liquid_volume.rs:111-199), in device memory:
// written by the host before a standalone advance, or filled in the carrier's
// step graph from the step's own dt, time and corrected faces.
struct LiquidFlowDev {
    const float* vel[3];
    const double* src;         // m^3/s per cell, or null
    double start, dt;
    rb200_liquid_stamp flow, inlet, source;
    double inlet_fraction[6];
    double max_courant, divergence_limit;
    int active;                // 0: nothing to do (the carrier step failed before the transport)
    int periodic;              // advance_periodic: seams instead of the inlet
};

// The state's bookkeeping (src/liquid_volume.rs:238-247), in device memory.
struct LiquidDev {
    double* frac[2];           // accepted = frac[acc]
    int acc;
    int pad;
    double time;
    unsigned long long id, version;
    double density, volume;
    double rh[3], rvolume;     // RN(1/h_d), RN(1/volume) where the fast division may use them, else 0
};

// Scratch of one advance.
struct LiquidScratch {
    double* part;
    unsigned* ticket;
    unsigned long long* first;  // [0] first failing cell, [1] first mismatched seam (axis << 40 | face)
    int* flags;
};

constexpr int kLiquidThreads = 256;

int liquid_blocks(const GridDev& g);
size_t liquid_partial_doubles(int blocks);
// Transport, reductions and the decision (report->error) for one interval;
// the accepted state is not replaced.
cudaError_t launch_liquid_advance(const GridDev& g, LiquidDev* L, const LiquidFlowDev* flow, const LiquidScratch& s,
                                  int blocks, rb200_liquid_report* report, cudaStream_t stream);
// Replace the accepted state by the candidate when the report accepts it.
cudaError_t launch_liquid_commit(LiquidDev* L, const rb200_liquid_report* report, cudaStream_t stream);

// LiquidVolumeState::new into device memory (h: host copy of *d; fraction
// host or device). RB200_LIQUID_REJECTED with *error filled on rejection.
int liquid_state_create(const GridDev& g, double density, rb200_liquid_stamp stamp, double time,
                        const double* fraction, uint64_t limit, LiquidDev* h, LiquidDev** d, LiquidScratch* sc,
                        int* blocks, rb200_liquid_report* error, cudaStream_t s);
void liquid_state_free(LiquidDev* h, LiquidDev* d, LiquidScratch* sc);

// Device side of the commit, for a caller that decides in its own kernel.
__device__ __forceinline__ void liquid_commit(LiquidDev* L, const rb200_liquid_report& r) {
    L->acc ^= 1;
    L->time = r.time;
    L->version = r.stamp.version;
}

}  // namespace rb200
