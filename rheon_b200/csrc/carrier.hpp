// Resident carrier state shared by the step graph (carrier.cu) and the
// host-driven forced step (sim_step.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "internal.hpp"
#include "liquid.hpp"
#include "pcg.hpp"

namespace rb200 {

constexpr int STEP_RUNNING = -1;

// Device-resident carrier descriptor (one per carrier).
struct CarrierDev {
    void* faces[3][3];   // [buffer][axis]
    float* tracer[2];
    int acc, tacc;       // accepted face buffer, accepted tracer
    int status;          // step status (STEP_RUNNING while the step runs)
    int skip;            // nonzero: skip the pressure solve (step already failed)
    int flags;           // validation flags of the step's kernels
    int pad;
    // step parameters (written by the host before each launch)
    double requested_dt, cfl, buoyancy;
    int iteration_limit_ok, skip_gates;
    int project_only;    // a projection: the accepted state is projected as supplied (no advection)
    int pad2;
    // configuration
    double max_courant, divergence_limit;
    // accepted-state bookkeeping
    double dt, rate, time;
    unsigned long long generation;
    double scalars[4];   // max|div|, max|u|, max|v|, max|w| of the corrected faces
    rb200_step_report report;
    int step_status;
    int trips;
    // AcceptedPreviousV1 initialization (src/pressure_initialization.rs:7-12)
    int warm_policy;     // configured policy
    int history;         // an accepted pressure of this state exists
    int warm;            // this step's solve is seeded
    double* accepted_p;  // the last accepted step's pressure (device)
    // liquid step (src/liquid_step.rs:828-900): null without a liquid state
    LiquidDev* liquid;
    LiquidFlowDev* lflow;
    rb200_liquid_report* lrep;
    unsigned long long flow_id;  // VolumeStamp id of the carrier's flow intervals
};

// Scratch of the host-driven forced step (sim_step.cu), made on its first use.
struct ForcedScratch;
void forced_scratch_free(ForcedScratch* scratch);

}  // namespace rb200

// Host side of the carrier (opaque handle of include/rheon_b200.h).
struct rb200_carrier {
    rb200_carrier_config cfg{};
    rb200::GridDev g{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t body_stream = nullptr;
    size_t elem = 4;
    void* faces[3][3] = {};
    float* tracer[2] = {nullptr, nullptr};
    double* accepted_p = nullptr;   // warm start: the last accepted pressure
    rb200::PcgSolver solver;
    rb200::CarrierDev* cd = nullptr;      // device
    rb200::CarrierDev* h_cd = nullptr;    // pinned host mirror
    cudaEvent_t ev[4] = {};
    cudaGraphExec_t step_exec = nullptr;
    int fixed_nodes = 0;
    size_t bytes = 0;
    bool in_flight = false;
    // liquid step state (rb200_carrier_attach_liquid)
    rb200::LiquidDev* lq_h = nullptr;   // pinned mirror, copied back after each step
    rb200::LiquidDev* lq_d = nullptr;
    rb200::LiquidFlowDev* lflow_h = nullptr;  // pinned: the per-step inputs
    rb200::LiquidFlowDev* lflow_d = nullptr;
    rb200_liquid_report* lrep_h = nullptr;  // pinned: the last step's liquid report
    rb200_liquid_report* lrep_d = nullptr;
    rb200::LiquidScratch lq_sc{};
    int lq_blocks = 0;
    bool lq_inputs = false;      // inlet and settings given
    uint64_t accepted_steps = 0;  // accepted steps since the last upload
    bool last_rejected = false;   // the last step was rejected
    std::string err;
    rb200::ForcedScratch* forced = nullptr;
    ~rb200_carrier() {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        rb200::forced_scratch_free(forced);
        if (step_exec) cudaGraphExecDestroy(step_exec);
        for (auto& b : faces)
            for (auto& a : b) cudaFree(a);
        cudaFree(tracer[0]);
        cudaFree(tracer[1]);
        cudaFree(accepted_p);
        if (lq_h) {
            rb200::liquid_state_free(lq_h, lq_d, &lq_sc);
            cudaFreeHost(lq_h);
        }
        cudaFree(lflow_d);
        cudaFree(lrep_d);
        if (lflow_h) cudaFreeHost(lflow_h);
        if (lrep_h) cudaFreeHost(lrep_h);
        cudaFree(cd);
        if (h_cd) cudaFreeHost(h_cd);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (stream) cudaStreamDestroy(stream);
    }
};

