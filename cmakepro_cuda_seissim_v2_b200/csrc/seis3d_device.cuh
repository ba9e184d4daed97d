// seis3d_device.cuh - device-side data layout and parameter blocks of the B200 solver.
//
// HBM layout (one session):
//   * 9 wavefields and 3 materials (1/rho, lambda, mu), each a padded X-contiguous volume
//     gx * gy * gz with the reference's ghost/CPML padding (cuda/Cuda_Seis3D.cu:459-462),
//     rows padded to a pitch that is a multiple of 32 elements (128 B in FP32) so every
//     row starts on a 128-byte line:  index(x,y,z) = z*plane + y*pitch + x.
//   * CPML memories psi only inside each axis's slab, six slots per axis (slots 0-2 are
//     written by the velocity pass, 3-5 by the stress pass), stored so that consecutive
//     x threads touch consecutive words on every axis:
//        x slab: psi0[slot][z][y][q]   q in [0, 2p)            (q runs along x)
//        y slab: psi1[slot][z][q][x]   q in [0, 2p), x pitched
//        z slab: psi2[slot][q][y][x]   q in [0, p or 2p), x pitched
//     (the reference's y/z slabs put the slab depth innermost, which strides adjacent x
//     threads by 2p words: cuda/Cuda_Seis3D.cu:104-106).
//   * CPML coefficient tables {a, b, 1/kappa} per axis node, centre then half grid
//     (cuda/Cuda_Seis3D.cu:45-64 layout).
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace seis3d {

constexpr int kRadius = 4;

// Geometry shared by every kernel of a session.
struct Geometry {
    int gx, gy, gz;
    int pml;
    int freeSurface;
    int reflecting;
    int thick[3];         // slab thickness per axis (2p, 2p, p or 2p)
    int64_t pitch;        // elements per row
    int64_t plane;        // elements per z plane
    float invH;           // 1 / spacing (IEEE, as 1.0f / c.spacing3D)
    float w[5];           // staggered weights w0..w3 and invH (a derivative is (sum w_r d_r) * invH)
    float h;
    float dt;
    double frequency;
    int ox, oy, oz;
    int nx, ny, nz;
    long long waitCycles;  // bound of every stage wait, in SM cycles
    int withheldStage;     // test hook: stage (plane index within a CTA's chunk) whose copies are
                           // never issued, so its wait runs out; -1 in normal operation
};

// Source parameters as the kernels consume them.
struct SourceParams {
    int gxs, gys, gzs;    // grid position of the centre node
    int kind;             // 0 explosion, 1 force
    float amplitude;
    float direction[3];
};

// Device clock and gather state shared by the kernels of one session.
struct Clock {
    unsigned long long step;   // time index of the step being executed
    int sample;                // samples recorded so far in the active gather
    int stride;                // gather stride (0 = no active gather)
    int target;                // samples to record
    int pad;
};

struct Fields {
    float* f[9];
    float* invRho;
    float* lambda;
    float* mu;
    float* psi[3];
    const float* coef[3];
    unsigned* status;          // [0] non-finite flag, [1] staging pipeline stall
    Clock* clock;
    const CUtensorMap* maps;   // TMA descriptors (tma::MapIndex), 64-byte aligned, global memory
};

}  // namespace seis3d
