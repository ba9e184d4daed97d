// Common.h - stand-in for the reference's Main_header/Common.h when its 2-D CUDA solver is
// compiled as a test oracle (TEST INFRASTRUCTURE ONLY).
//
// The reference header also declares the application's OpenGL/GLFW/ImGui state, which this
// headless build does not need and which the image has no headers for.  CUDA_Kernels/Cuda_Check.cu
// only uses the solver types below, so this file declares exactly those, written from the
// reference's field lists so that the memory layout is the same:
//   GPUSource          Main_header/Common.h:251-256
//   SimulationContext  Main_header/Common.h:259-287
//   ReplayManager      Main_header/Common.h:320-330 (frames and the upload member only)
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846f
#endif

struct GPUSource {
    int idx;
    float t;
    float f_peak;
    float amp;
};

struct SimulationContext {
    int NX, NZ;
    int total_grid;
    float h, dt;
    int nt, npml;
    int snap_spacenum;
    int flag_type;
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

struct ReplayManager {
    std::vector<std::vector<float>> frames;
    void uploadFrameToGpu(int frameIdx, GPUSimData& gpu);
};
