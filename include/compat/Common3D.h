// Common3D.h - the namespace Seis3D types of the SeisWave Lab 3-D solver API, for code that is
// compiled unchanged against the B200 solver (include/seis3d_capi.h).
//
// Types and member names follow the reference header include/Common3D.h (constants :9-16,
// enums :18-22, SimulationContext3D :24-42, Source3D :44-49, Receiver3D :51, ViewLayout3D
// :53-60, MemoryBudget3D :72-74, GPUSimData3D :76-93, gridIndex3D :96-98), because callers
// name them.  The defaults of SimulationContext3D and Source3D are taken from the library
// (seis3d_default_context / seis3d_default_source) rather than repeated here.
//
// GPUSimData3D carries two members the reference does not have: the opaque session handle
// (session3D) and the row pitch of the device fields (pitch3D).  Sessions created through
// Cuda_Seis3D.cuh use the reference's unpitched rows (pitch3D == gx3D) whenever gx3D is a
// multiple of 4, which is what code indexing field3D[] directly expects.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>

#include "../seis3d_capi.h"

namespace Seis3D {

constexpr int stencilRadius3D = SEIS3D_STENCIL_RADIUS;
constexpr std::size_t maxPhysicalNodes3D = SEIS3D_MAX_PHYSICAL_NODES;
constexpr int maxVolumeAxis3D = SEIS3D_MAX_VOLUME_AXIS;
constexpr int maxVolumeOutput3D = SEIS3D_MAX_VOLUME_OUTPUT;
constexpr std::size_t memoryLimit3D = SEIS3D_MEMORY_LIMIT;
constexpr int maxReceivers3D = SEIS3D_MAX_RECEIVERS;
constexpr int maxSegySamples3D = SEIS3D_MAX_SEGY_SAMPLES;
constexpr int maxSegyIntervalUs3D = SEIS3D_MAX_SEGY_INTERVAL_US;

enum class Field3D : int { Vx, Vy, Vz, Sxx, Syy, Szz, Sxy, Syz, Sxz };
enum class ModelKind3D : int { Uniform, TwoLayer, Sphere, Imported, ThreeLayer, DippingLayer,
                               LowVelocityLayer, Fault, Gradient, SaltDome };
enum class SourceKind3D : int { Explosion, Force };

struct SimulationContext3D {
    int nx3D, ny3D, nz3D;
    int pml3D;
    bool freeSurface3D;
    bool reflecting3D;
    float spacing3D, cfl3D, dt3D;
    bool manualTimeStep3D;
    float requestedDtMs3D;
    float safeDt3D;
    float vp3D, vs3D, density3D;
    float layerVp3D, layerVs3D, layerDensity3D;
    float maxVp3D, frequency3D;
    ModelKind3D modelKind3D;
    float interfaceDepth3D, layerDip3D, layerThickness3D;
    float faultThrow3D, anomalyRadius3D;
    int gx3D, gy3D, gz3D, ox3D, oy3D, oz3D;
    std::size_t cells3D;

    SimulationContext3D() {
        seis3d_context c;
        seis3d_default_context(&c);
        assign(c);
    }
    explicit SimulationContext3D(const seis3d_context& c) { assign(c); }

    void assign(const seis3d_context& c) {
        nx3D = c.nx3D; ny3D = c.ny3D; nz3D = c.nz3D; pml3D = c.pml3D;
        freeSurface3D = c.freeSurface3D != 0; reflecting3D = c.reflecting3D != 0;
        spacing3D = c.spacing3D; cfl3D = c.cfl3D; dt3D = c.dt3D;
        manualTimeStep3D = c.manualTimeStep3D != 0; requestedDtMs3D = c.requestedDtMs3D; safeDt3D = c.safeDt3D;
        vp3D = c.vp3D; vs3D = c.vs3D; density3D = c.density3D;
        layerVp3D = c.layerVp3D; layerVs3D = c.layerVs3D; layerDensity3D = c.layerDensity3D;
        maxVp3D = c.maxVp3D; frequency3D = c.frequency3D; modelKind3D = ModelKind3D(c.modelKind3D);
        interfaceDepth3D = c.interfaceDepth3D; layerDip3D = c.layerDip3D; layerThickness3D = c.layerThickness3D;
        faultThrow3D = c.faultThrow3D; anomalyRadius3D = c.anomalyRadius3D;
        gx3D = c.gx3D; gy3D = c.gy3D; gz3D = c.gz3D; ox3D = c.ox3D; oy3D = c.oy3D; oz3D = c.oz3D;
        cells3D = std::size_t(c.cells3D);
    }

    seis3d_context toC() const {
        seis3d_context c{};
        c.nx3D = nx3D; c.ny3D = ny3D; c.nz3D = nz3D; c.pml3D = pml3D;
        c.freeSurface3D = freeSurface3D; c.reflecting3D = reflecting3D;
        c.spacing3D = spacing3D; c.cfl3D = cfl3D; c.dt3D = dt3D;
        c.manualTimeStep3D = manualTimeStep3D; c.requestedDtMs3D = requestedDtMs3D; c.safeDt3D = safeDt3D;
        c.vp3D = vp3D; c.vs3D = vs3D; c.density3D = density3D;
        c.layerVp3D = layerVp3D; c.layerVs3D = layerVs3D; c.layerDensity3D = layerDensity3D;
        c.maxVp3D = maxVp3D; c.frequency3D = frequency3D; c.modelKind3D = int(modelKind3D);
        c.interfaceDepth3D = interfaceDepth3D; c.layerDip3D = layerDip3D; c.layerThickness3D = layerThickness3D;
        c.faultThrow3D = faultThrow3D; c.anomalyRadius3D = anomalyRadius3D;
        c.gx3D = gx3D; c.gy3D = gy3D; c.gz3D = gz3D; c.ox3D = ox3D; c.oy3D = oy3D; c.oz3D = oz3D;
        c.cells3D = uint64_t(cells3D);
        return c;
    }
};

struct Source3D {
    int x3D, y3D, z3D;
    SourceKind3D kind3D;
    float amplitude3D;
    float direction3D[3];

    Source3D() {
        seis3d_source s;
        seis3d_default_source(&s);
        x3D = s.x3D; y3D = s.y3D; z3D = s.z3D; kind3D = SourceKind3D(s.kind3D); amplitude3D = s.amplitude3D;
        for (int a = 0; a < 3; ++a) direction3D[a] = s.direction3D[a];
    }
    seis3d_source toC() const {
        seis3d_source s{};
        s.x3D = x3D; s.y3D = y3D; s.z3D = z3D; s.kind3D = int(kind3D); s.amplitude3D = amplitude3D;
        for (int a = 0; a < 3; ++a) s.direction3D[a] = direction3D[a];
        return s;
    }
};

struct Receiver3D { int x3D = 0, y3D = 0, z3D = 0; };
static_assert(sizeof(Receiver3D) == sizeof(seis3d_receiver), "Receiver3D is passed to the C ABI as is");

struct ViewLayout3D {
    std::size_t sliceOffset3D[3]{};
    int sliceWidth3D[3]{}, sliceHeight3D[3]{};
    std::size_t volumeOffset3D = 0, totalSamples3D = 0;
    int volumeX3D = 0, volumeY3D = 0, volumeZ3D = 0;
    int domainSize3D[3]{}, domainOrigin3D[3]{};
};

// activePml3D / boundaryName3D of the reference header.
__host__ __device__ inline int activePml3D(const SimulationContext3D& c) { return c.reflecting3D ? 0 : c.pml3D; }
inline const char* boundaryName3D(const SimulationContext3D& c) {
    return c.reflecting3D ? "Reflecting slip walls" : c.freeSurface3D ? "Free top + CPML" : "All faces CPML";
}

struct MemoryBudget3D {
    std::size_t fieldBytes3D = 0, cpmlBytes3D = 0, viewBytes3D = 0, totalBytes3D = 0;
};

struct GPUSimData3D {
    float* field3D[9]{};
    float* inverseDensity3D = nullptr;
    float* lambda3D = nullptr;
    float* mu3D = nullptr;
    float* cpml3D[3]{};
    std::size_t slabCells3D[3]{};
    float* coefficients3D[3]{};
    Receiver3D* receivers3D = nullptr;
    float* receiverValues3D = nullptr;
    float* hostReceiverValues3D = nullptr;
    unsigned int* viewStatistics3D = nullptr;
    cudaStream_t stream3D = nullptr;
    cudaEvent_t startEvent3D = nullptr, stopEvent3D = nullptr;
    int receiverCount3D = 0;
    std::size_t allocatedBytes3D = 0;
    seis3d_session* session3D = nullptr;  // B200 solver session (not in the reference struct)
    std::int64_t pitch3D = 0;             // elements per device row (== gx3D in the unpitched layout)
};

inline std::size_t gridIndex3D(const SimulationContext3D& c, int x, int y, int z) {
    return (std::size_t(z) * c.gy3D + y) * c.gx3D + x;
}

}  // namespace Seis3D
