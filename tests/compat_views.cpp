// A C++ caller of the header-only reference layer (include/compat/Cuda_Seis3D.cuh) that draws
// views the way the reference's renderer does (src/Seis3D/Renderer3D.cpp:192): it runs a small
// shot through the Seis3D:: functions, calls Seis3D::extractViews3D into a device buffer, and
// checks the result against the C entry point seis3d_extract_views on the same session.
// Compiled by tests/test_compat_views.py.  Exit status: 0 when both calls agree bit for bit,
// 1 on a mismatch, 2 on an exception, 77 without a GPU.
#include "Cuda_Seis3D.cuh"

#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

int main() {
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return 77;
    try {
        Seis3D::SimulationContext3D context;
        context.nx3D = 48; context.ny3D = 40; context.nz3D = 44; context.pml3D = 8;
        Seis3D::validateContext3D(context);
        Seis3D::GPUSimData3D gpu;
        Seis3D::initializeGpu3D(gpu, context);
        Seis3D::Source3D source;
        source.x3D = 24; source.y3D = 20; source.z3D = 12;
        for (std::uint64_t n = 0; n < 30; ++n) Seis3D::runStep3D(gpu, context, source, n);
        const Seis3D::ViewLayout3D layout = Seis3D::makeViewLayout3D(context);
        const std::size_t floats = layout.totalSamples3D * 2;
        float* a = nullptr;
        float* b = nullptr;
        if (cudaMalloc(&a, floats * sizeof(float)) != cudaSuccess || cudaMalloc(&b, floats * sizeof(float)) != cudaSuccess)
            return 2;
        const int slices[3] = {24, 20, 12};
        float maximum = 0.0f, range[2] = {0.0f, 0.0f}, velocityMaximum = 0.0f;
        Seis3D::extractViews3D(gpu, context, a, layout, slices, 0, 5, true, maximum, range, false, &velocityMaximum);
        const seis3d_context c = context.toC();
        seis3d_view_layout l{};
        Seis3D::compat3D::check(seis3d_make_view_layout(&c, &l));
        float maximum2 = 0.0f, range2[2] = {0.0f, 0.0f}, velocityMaximum2 = 0.0f;
        Seis3D::compat3D::check(seis3d_extract_views(gpu.session3D, &c, b, &l, slices, 0, 5, 1, 0, &maximum2, range2,
                                                     &velocityMaximum2));
        std::vector<float> ha(floats), hb(floats);
        if (cudaMemcpy(ha.data(), a, floats * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(hb.data(), b, floats * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            return 2;
        cudaFree(a);
        cudaFree(b);
        Seis3D::releaseGpu3D(gpu);
        const bool same = std::memcmp(ha.data(), hb.data(), floats * sizeof(float)) == 0 && maximum == maximum2 &&
                          range[0] == range2[0] && range[1] == range2[1] && velocityMaximum == velocityMaximum2;
        std::printf("views %zu maximum %.9g velocity %.9g material %.9g %.9g\n", layout.totalSamples3D, maximum,
                    velocityMaximum, range[0], range[1]);
        return same && maximum > 0.0f ? 0 : 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
}
