// seis3d_oracle_gpu.cu - FP64 restatement of the reference scheme on the GPU.
//
// TEST INFRASTRUCTURE ONLY (the oracle role): the same scheme as the FP64 path of
// seis3d_oracle.cpp (cuda/Cuda_Seis3D.cu:78-111 derivatives and CPML, :203-219 and :249-272
// free-surface images, :222-245 velocity, :275-310 stress, :313-332 source, :335-352
// receivers, :602-624 step order) with one GPU thread per cell and every value in double, so
// that the full-size workloads (300 x 300 x 400, 2500 steps) get an FP64 answer in seconds
// instead of the CPU oracle's hours.  It is plain code on purpose (global loads, no staging):
// it is the yardstick of the FP32 kernels, not a product path.  Validation, CPML profiles and
// slab sizes come from the CPU oracle's host code, included below.
#define SEIS3D_ORACLE_HOST_ONLY
#include "seis3d_oracle.cpp"

#include <cuda_runtime.h>

#include <memory>
#include <stdexcept>

namespace {

struct Dev {
    int gx, gy, gz, pml, freeSurface;
    long long sy, sz;
    double* f[9];
    double *invRho, *lambda, *mu;
    double* psi[3];
    long long slab[3];
    const double* coef[3];
    double inv, dt, h;
};

__device__ __forceinline__ double wd(int r) {
    return r == 0 ? 1225.0 / 1024.0 : r == 1 ? -245.0 / 3072.0 : r == 2 ? 49.0 / 5120.0 : -5.0 / 7168.0;
}

template <bool plus> __device__ double diffD(const double* f, long long i, long long st, double inv) {
    double sum = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) sum += wd(r) * (f[i + (r + (plus ? 1 : 0)) * st] - f[i - (r + (plus ? 0 : 1)) * st]);
    return sum * inv;
}

__device__ double cpmlD(const Dev& D, int x, int y, int z, int axis, int slot, bool half, double d) {
    const int n = axis == 0 ? D.gx : axis == 1 ? D.gy : D.gz;
    const int coord = axis == 0 ? x : axis == 1 ? y : z;
    const bool topFree = axis == 2 && D.freeSurface;
    int q = -1;
    if (!topFree && coord < kRadius + D.pml) q = coord - kRadius;
    else if (coord >= n - kRadius - D.pml) q = (topFree ? 0 : D.pml) + coord - (n - kRadius - D.pml);
    if (q < 0) return d;
    const int thick = (topFree ? 1 : 2) * D.pml;
    const long long s = axis == 0 ? ((long long)z * D.gy + y) * thick + q
                      : axis == 1 ? ((long long)z * D.gx + x) * thick + q
                                  : ((long long)y * D.gx + x) * thick + q;
    double& m = D.psi[axis][slot * D.slab[axis] + s];
    const double* k = D.coef[axis] + ((long long)(half ? 1 : 0) * n + coord) * 3;
    const double updated = k[1] * m + k[0] * d;
    m = updated;
    return k[2] * d + updated;
}

__device__ __forceinline__ long long idx(const Dev& D, int x, int y, int z) { return (z * (long long)D.gy + y) * D.gx + x; }

__global__ void stressGhostsD(Dev D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 4, y = blockIdx.y * blockDim.y + threadIdx.y + 4;
    if (x >= D.gx - 4 || y >= D.gy - 4) return;
    D.f[5][idx(D, x, y, 4)] = 0;
    for (int k = 1; k <= 4; ++k) {
        const long long g = idx(D, x, y, 4 - k), m = idx(D, x, y, 4 + k), sm = idx(D, x, y, 3 + k);
        D.f[5][g] = -D.f[5][m];
        D.f[8][g] = -D.f[8][sm];
        D.f[7][g] = -D.f[7][sm];
        D.f[3][g] = D.f[3][m];
        D.f[4][g] = D.f[4][m];
        D.f[6][g] = D.f[6][m];
    }
}

__global__ void velocityD(Dev D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 4, y = blockIdx.y + 4, z = blockIdx.z + 4;
    if (x >= D.gx - 4) return;
    const long long i = idx(D, x, y, z);
    const long long st[3] = {1, D.sy, D.sz};
    const int S[3][3] = {{3, 6, 8}, {6, 4, 7}, {8, 7, 5}};
    for (int v = 0; v < 3; ++v) {
        double div = 0;
        for (int a = 0; a < 3; ++a) {
            const double* f = D.f[S[v][a]];
            const double d = a == v ? diffD<true>(f, i, st[a], D.inv) : diffD<false>(f, i, st[a], D.inv);
            div += cpmlD(D, x, y, z, a, v, a == v, d);
        }
        const double A = D.invRho[i], B = D.invRho[i + st[v]];
        D.f[v][i] = D.f[v][i] + D.dt * (2 * A * B / (A + B)) * div;
    }
}

__global__ void velocityGhostsD(Dev D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 4, y = blockIdx.y * blockDim.y + threadIdx.y + 4;
    if (x >= D.gx - 4 || y >= D.gy - 4) return;
    const long long i = idx(D, x, y, 4), next = i + D.sz;
    const double ex = diffD<false>(D.f[0], i, 1, D.inv);
    const double ey = diffD<false>(D.f[1], i, D.sy, D.inv);
    const double dzVx = -(1.5 * diffD<true>(D.f[2], i, 1, D.inv) - 0.5 * diffD<true>(D.f[2], next, 1, D.inv));
    const double dzVy = -(1.5 * diffD<true>(D.f[2], i, D.sy, D.inv) - 0.5 * diffD<true>(D.f[2], next, D.sy, D.inv));
    const double dzVz = -D.lambda[i] / (D.lambda[i] + 2 * D.mu[i]) * (ex + ey);
    for (int k = 1; k <= 4; ++k) {
        const long long g = idx(D, x, y, 4 - k), m = idx(D, x, y, 4 + k);
        D.f[0][g] = D.f[0][m] - double(2 * k) * D.h * dzVx;
        D.f[1][g] = D.f[1][m] - double(2 * k) * D.h * dzVy;
        D.f[2][g] = D.f[2][idx(D, x, y, 3 + k)] - double(2 * k - 1) * D.h * dzVz;
    }
}

__device__ double shearMuD(const Dev& D, long long i, long long a, long long b) {
    const double m0 = D.mu[i], m1 = D.mu[i + a], m2 = D.mu[i + b], m3 = D.mu[i + a + b];
    return (m0 > 0 && m1 > 0 && m2 > 0 && m3 > 0) ? 4 / (1 / m0 + 1 / m1 + 1 / m2 + 1 / m3) : 0.0;
}

__global__ void stressD(Dev D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 4, y = blockIdx.y + 4, z = blockIdx.z + 4;
    if (x >= D.gx - 4) return;
    const long long i = idx(D, x, y, z);
    const long long st[3] = {1, D.sy, D.sz};
    double d[3][3];
    for (int v = 0; v < 3; ++v)
        for (int a = 0; a < 3; ++a) {
            const double raw = a == v ? diffD<false>(D.f[v], i, st[a], D.inv) : diffD<true>(D.f[v], i, st[a], D.inv);
            d[v][a] = cpmlD(D, x, y, z, a, 3 + v, a != v, raw);
        }
    const double L = D.lambda[i], M = D.mu[i];
    const bool top = D.freeSurface && z == 4;
    if (top) d[2][2] = -L / (L + 2 * M) * (d[0][0] + d[1][1]);
    const double tr = d[0][0] + d[1][1] + d[2][2];
    D.f[3][i] += D.dt * (L * tr + 2 * M * d[0][0]);
    D.f[4][i] += D.dt * (L * tr + 2 * M * d[1][1]);
    D.f[5][i] = top ? 0.0 : D.f[5][i] + D.dt * (L * tr + 2 * M * d[2][2]);
    D.f[6][i] += D.dt * shearMuD(D, i, st[0], st[1]) * (d[0][1] + d[1][0]);
    D.f[7][i] += D.dt * shearMuD(D, i, st[1], st[2]) * (d[1][2] + d[2][1]);
    D.f[8][i] += D.dt * shearMuD(D, i, st[0], st[2]) * (d[0][2] + d[2][0]);
}

struct SourceD { int gxs, gys, gzs, kind; double amplitude, direction[3], frequency; };

__global__ void sourceKernelD(Dev D, SourceD S, double time) {
    const int a = threadIdx.x;
    if (a >= 27) return;
    const int dx = a % 3 - 1, dy = (a / 3) % 3 - 1, dz = a / 9 - 1;
    const long long i = idx(D, S.gxs + dx, S.gys + dy, S.gzs + dz);
    const double phase = 3.141592653589793 * S.frequency * (time - 1.2 / S.frequency);
    const double ricker = (1 - 2 * phase * phase) * exp(-phase * phase);
    const double norm = pow(1.0 + 2.0 * exp(-0.5), 3.0);
    const double value = D.dt * S.amplitude * ricker * exp(-0.5 * double(dx * dx + dy * dy + dz * dz)) / norm;
    if (S.kind == SEIS3D_SOURCE_EXPLOSION) {
        D.f[3][i] += value; D.f[4][i] += value; D.f[5][i] += value;
    } else {
        const long long st[3] = {1, D.sy, D.sz};
        for (int v = 0; v < 3; ++v) {
            const double A = D.invRho[i], B = D.invRho[i + st[v]];
            D.f[v][i] += value * S.direction[v] * (2 * A * B / (A + B));
        }
    }
}

__global__ void sampleD(Dev D, const int3* r, int count, double* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const long long i = idx(D, r[k].x, r[k].y, r[k].z);
    out[3 * k + 0] = 0.5 * (D.f[0][i] + D.f[0][i - 1]);
    out[3 * k + 1] = 0.5 * (D.f[1][i] + D.f[1][i - D.sy]);
    out[3 * k + 2] = 0.5 * (D.f[2][i] + D.f[2][i - D.sz]);
}

// Materials from FP32 SI volumes [z][y][x] (the FP64 formulas of setMaterial), then the
// nearest physical cell copied into padding (cuda/Cuda_Seis3D.cu:188-200).
__global__ void materialsD(Dev D, const float* vp, const float* vs, const float* rho, int nx, int ny, int nz, int ox,
                           int oy, int oz) {
    const long long n = (long long)D.gx * D.gy * D.gz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = int(i % D.gx), y = int((i / D.gx) % D.gy), z = int(i / ((long long)D.gx * D.gy));
    const int px = min(max(x - ox, 0), nx - 1), py = min(max(y - oy, 0), ny - 1), pz = min(max(z - oz, 0), nz - 1);
    const long long k = ((long long)pz * ny + py) * nx + px;
    const double P = vp[k], S = vs[k], R = rho[k];
    D.invRho[i] = 1.0 / R;
    D.mu[i] = R * S * S;
    D.lambda[i] = R * (P * P - 2.0 * S * S);
}

}  // namespace

namespace {

struct GpuOracle {
    seis3d_context c{};
    Dev D{};
    double* pool = nullptr;
    int3* receivers = nullptr;
    int receiverCount = 0;
    double* samples = nullptr;
    std::vector<double*> owned;

    ~GpuOracle() {
        cudaDeviceSynchronize();
        for (double* p : owned) cudaFree(p);
        cudaFree(pool);
        cudaFree(receivers);
        cudaFree(samples);
    }
    double* alloc(std::size_t n) {
        double* p = nullptr;
        if (cudaMalloc(&p, std::max<std::size_t>(n, 1) * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("FP64 oracle: device allocation failed");
        cudaMemset(p, 0, std::max<std::size_t>(n, 1) * sizeof(double));
        owned.push_back(p);
        return p;
    }
    void step(const seis3d_source& s, uint64_t n) {
        const dim3 plane((c.gx3D - 8 + 31) / 32, (c.gy3D - 8 + 7) / 8), planeBlock(32, 8);
        const dim3 cells((c.gx3D - 8 + 127) / 128, c.gy3D - 8, c.gz3D - 8);
        SourceD S{};
        S.gxs = s.x3D + c.ox3D; S.gys = s.y3D + c.oy3D; S.gzs = s.z3D + c.oz3D;
        S.kind = s.kind3D; S.amplitude = s.amplitude3D; S.frequency = c.frequency3D;
        for (int a = 0; a < 3; ++a) S.direction[a] = s.direction3D[a];
        if (c.freeSurface3D) stressGhostsD<<<plane, planeBlock>>>(D);
        velocityD<<<cells, 128>>>(D);
        if (s.kind3D == SEIS3D_SOURCE_FORCE) sourceKernelD<<<1, 32>>>(D, S, double(n) * double(c.dt3D));
        if (c.freeSurface3D) velocityGhostsD<<<plane, planeBlock>>>(D);
        stressD<<<cells, 128>>>(D);
        if (s.kind3D == SEIS3D_SOURCE_EXPLOSION) sourceKernelD<<<1, 32>>>(D, S, (double(n) + 0.5) * double(c.dt3D));
        if (c.freeSurface3D) stressGhostsD<<<plane, planeBlock>>>(D);
    }
};

thread_local std::string gpuMessage;

template <class F> int guard(F&& body) {
    try {
        body();
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
        return 0;
    } catch (const std::exception& e) {
        gpuMessage = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

const char* oracle3d_gpu_last_error(void) { return gpuMessage.c_str(); }

// A zeroed FP64 state for a validated context (CPML 4..40 accepted).
void* oracle3d_gpu_create(const seis3d_context* context) {
    GpuOracle* o = nullptr;
    const int status = guard([&] {
        seis3d_context c = *context;
        const int saved = g_minPml;
        g_minPml = 4;
        const std::string msg = validate(c);
        g_minPml = saved;
        if (!msg.empty()) throw std::runtime_error(msg);
        if (c.reflecting3D) throw std::runtime_error("FP64 oracle: reflecting walls are not restated on the GPU");
        auto g = std::make_unique<GpuOracle>();
        g->c = c;
        Dev& D = g->D;
        D.gx = c.gx3D; D.gy = c.gy3D; D.gz = c.gz3D; D.pml = c.pml3D; D.freeSurface = c.freeSurface3D;
        D.sy = c.gx3D; D.sz = (long long)c.gx3D * c.gy3D;
        D.inv = 1.0 / double(c.spacing3D);
        D.dt = double(c.dt3D);
        D.h = double(c.spacing3D);
        const std::size_t cells = std::size_t(c.cells3D);
        for (int k = 0; k < 9; ++k) D.f[k] = g->alloc(cells);
        D.invRho = g->alloc(cells); D.lambda = g->alloc(cells); D.mu = g->alloc(cells);
        for (int a = 0; a < 3; ++a) {
            D.slab[a] = (long long)slabCells(c, a);
            D.psi[a] = g->alloc(std::size_t(D.slab[a]) * 6);
            const auto p = profile(c, a);
            double* k = g->alloc(p.size());
            cudaMemcpy(k, p.data(), p.size() * sizeof(double), cudaMemcpyHostToDevice);
            D.coef[a] = k;
        }
        o = g.release();
    });
    return status == 0 ? o : nullptr;
}

void oracle3d_gpu_destroy(void* h) { delete static_cast<GpuOracle*>(h); }

// vp, vs, rho: host FP32 volumes [nz][ny][nx] of the physical model.
int oracle3d_gpu_upload_model(void* h, const float* vp, const float* vs, const float* rho) {
    auto* o = static_cast<GpuOracle*>(h);
    return guard([&] {
        const seis3d_context& c = o->c;
        const std::size_t n = std::size_t(c.nx3D) * c.ny3D * c.nz3D;
        float* d = nullptr;
        if (cudaMalloc(&d, 3 * n * sizeof(float)) != cudaSuccess) throw std::runtime_error("FP64 oracle: upload buffer");
        cudaMemcpy(d, vp, n * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(d + n, vs, n * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(d + 2 * n, rho, n * sizeof(float), cudaMemcpyHostToDevice);
        const long long cells = (long long)c.cells3D;
        materialsD<<<unsigned((cells + 255) / 256), 256>>>(o->D, d, d + n, d + 2 * n, c.nx3D, c.ny3D, c.nz3D, c.ox3D,
                                                           c.oy3D, c.oz3D);
        cudaDeviceSynchronize();
        cudaFree(d);
    });
}

int oracle3d_gpu_set_receivers(void* h, const seis3d_receiver* r, int count) {
    auto* o = static_cast<GpuOracle*>(h);
    return guard([&] {
        std::vector<int3> p(std::max(count, 1));
        for (int k = 0; k < count; ++k) p[k] = make_int3(r[k].x3D + o->c.ox3D, r[k].y3D + o->c.oy3D, r[k].z3D + o->c.oz3D);
        cudaFree(o->receivers);
        cudaFree(o->samples);
        o->receivers = nullptr;
        o->samples = nullptr;
        if (cudaMalloc(&o->receivers, p.size() * sizeof(int3)) != cudaSuccess ||
            cudaMalloc(&o->samples, p.size() * 3 * sizeof(double)) != cudaSuccess)
            throw std::runtime_error("FP64 oracle: receiver buffers");
        cudaMemcpy(o->receivers, p.data(), p.size() * sizeof(int3), cudaMemcpyHostToDevice);
        o->receiverCount = count;
    });
}

// `count` steps from `first`; after every step with (n + 1) % stride == 0 the receivers are
// sampled into out ([sample][receiver][3], at most `capacity` samples).
int oracle3d_gpu_run_gather(void* h, const seis3d_source* s, uint64_t first, int count, int stride, double* out,
                            int capacity, int* taken) {
    auto* o = static_cast<GpuOracle*>(h);
    *taken = 0;
    return guard([&] {
        const std::size_t per = std::size_t(o->receiverCount) * 3;
        for (int k = 0; k < count; ++k) {
            const uint64_t n = first + uint64_t(k);
            o->step(*s, n);
            if (stride > 0 && (n + 1) % uint64_t(stride) == 0 && *taken < capacity && o->receiverCount > 0) {
                sampleD<<<(o->receiverCount + 127) / 128, 128>>>(o->D, o->receivers, o->receiverCount, o->samples);
                cudaMemcpy(out + std::size_t(*taken) * per, o->samples, per * sizeof(double), cudaMemcpyDeviceToHost);
                ++*taken;
            }
        }
        cudaDeviceSynchronize();
    });
}

int oracle3d_gpu_get_field(void* h, int k, double* out) {
    auto* o = static_cast<GpuOracle*>(h);
    return guard([&] {
        if (k < 0 || k > 8) throw std::runtime_error("FP64 oracle: field index");
        cudaMemcpy(out, o->D.f[k], std::size_t(o->c.cells3D) * sizeof(double), cudaMemcpyDeviceToHost);
    });
}

}  // extern "C"
