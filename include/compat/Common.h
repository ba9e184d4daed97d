// Common.h - the 2-D solver types of the SeisWave Lab API (Main_header/Common.h:251-330:
// GPUSource, SimulationContext, ReplayManager) for code compiled unchanged against the B200
// solver.  Only the solver types are declared: the application's window, UI and OpenGL
// state of the reference header are not part of this library.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../seis2d_capi.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

// One active source of the multi-source array (same layout as seis2d_source).
struct GPUSource {
    int idx;
    float t;
    float f_peak;
    float amp;
};
static_assert(sizeof(GPUSource) == sizeof(seis2d_source), "GPUSource is copied to the device as is");

struct SimulationContext {
    int NX, NZ;
    int total_grid;
    float h, dt;
    int nt, npml;
    int snap_spacenum;
    int flag_type;  // 1 split-field PML, 2 hybrid, 3 free surface

    std::vector<float> rho, mu, lambda, lambda2mu;
    std::vector<float> dp_flat;
    std::vector<float> dx, dx_half, dz, dz_half;

    float c1_h, c2_h, c3_h, c4_h;

    int src_idx;
    int src_z_idx;
    std::vector<float> wavelet;
    float src_angle;
    int src_type;
    float src_amp;

    int num_rcv;
    std::vector<int> rcv_grid_idx;

    std::vector<float> record_vx;
    std::vector<float> record_vz;

    bool upFlag;
};

struct GPUSimData;

// Host cache of wavefield frames for replay.
struct ReplayManager {
    int maxFrames = 500;
    int recordStride = 5;
    float playbackSpeed = 1.0f;
    int currentFrameIndex = 0;
    float currentFrameFloat = 0.0f;
    std::vector<std::vector<float>> frames;

    void clear() {
        frames.clear();
        currentFrameIndex = 0;
        currentFrameFloat = 0.0f;
    }
    // Restores frame `frameIdx` into the vertical velocity of the solver (defined in
    // Cuda_Check.cuh, which completes GPUSimData).
    void uploadFrameToGpu(int frameIdx, GPUSimData& gpu);
};
