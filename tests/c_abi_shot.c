/* A plain C99 caller of the two solver libraries, compiled by tests/test_c_abi.py: it proves
 * that the headers are C (not C++) and that every call it makes is exported, and on a GPU it
 * runs a small 3-D shot (procedural model, device gather, checkpoint round trip) and a small
 * 2-D shot, printing one line of numbers for the test to check.  Exit status: 0 on success,
 * 2 for an API error (message on stderr). */
#include "seis2d_capi.h"
#include "seis3d_capi.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define CHECK3(call)                                                                   \
    do {                                                                               \
        if ((call) != SEIS3D_OK) {                                                     \
            fprintf(stderr, "%s failed: %s\n", #call, seis3d_last_error());            \
            return 2;                                                                  \
        }                                                                              \
    } while (0)

#define CHECK2(call)                                                                   \
    do {                                                                               \
        if ((call) != SEIS2D_OK) {                                                     \
            fprintf(stderr, "%s failed: %s\n", #call, seis2d_last_error());            \
            return 2;                                                                  \
        }                                                                              \
    } while (0)

static double norm(const float* v, size_t n) {
    double s = 0.0;
    size_t i;
    for (i = 0; i < n; ++i) s += (double)v[i] * v[i];
    return sqrt(s);
}

static int shot3d(double* gatherNorm, int* restartExact) {
    seis3d_context c;
    seis3d_source src;
    seis3d_session* s = NULL;
    seis3d_session* t = NULL;
    seis3d_receiver rec[4];
    float gather[40 * 4 * 3], again[40 * 4 * 3];
    unsigned char* state;
    uint64_t bytes = 0;
    int taken = 0, i;

    seis3d_default_context(&c);
    c.nx3D = 40; c.ny3D = 32; c.nz3D = 36; c.pml3D = 8;
    CHECK3(seis3d_validate_context(&c));
    seis3d_default_source(&src);
    src.x3D = 20; src.y3D = 16; src.z3D = 10;
    for (i = 0; i < 4; ++i) { rec[i].x3D = 5 + 8 * i; rec[i].y3D = 16; rec[i].z3D = 0; }
    CHECK3(seis3d_initialize(&s, &c, NULL));
    CHECK3(seis3d_set_receivers(s, &c, rec, 4));
    CHECK3(seis3d_run_steps(s, &c, &src, 0, 20));
    CHECK3(seis3d_checkpoint_bytes(s, &bytes));
    state = (unsigned char*)malloc((size_t)bytes);
    if (!state) return 2;
    CHECK3(seis3d_save_checkpoint(s, state, bytes));
    CHECK3(seis3d_gather_begin(s, 1, 40));
    CHECK3(seis3d_run_steps(s, &c, &src, 20, 40));
    CHECK3(seis3d_gather_fetch(s, gather, sizeof(gather) / sizeof(float), &taken));
    *gatherNorm = taken == 40 ? norm(gather, sizeof(gather) / sizeof(float)) : -1.0;
    /* A second session restarted from the checkpoint records the same gather. */
    CHECK3(seis3d_initialize(&t, &c, NULL));
    CHECK3(seis3d_set_receivers(t, &c, rec, 4));
    CHECK3(seis3d_load_checkpoint(t, state, bytes));
    CHECK3(seis3d_gather_begin(t, 1, 40));
    CHECK3(seis3d_run_steps(t, &c, &src, 20, 40));
    CHECK3(seis3d_gather_fetch(t, again, sizeof(again) / sizeof(float), &taken));
    *restartExact = 1;
    for (i = 0; i < 40 * 4 * 3; ++i)
        if (gather[i] != again[i]) *restartExact = 0;
    free(state);
    seis3d_release(s);
    seis3d_release(t);
    return 0;
}

static int shot2d(double* traceNorm) {
    enum { N = 96, NT = 200 };
    static float rho[N * N], mu[N * N], lam[N * N], l2m[N * N], dp[N], dx[N], dxh[N], dz[N], dzh[N], wavelet[NT];
    static float vx[NT], vz[NT];
    double w[4];
    int rcv = (N / 2) * N + N / 2 + 8, i, taken = 0;
    seis2d_context c;
    seis2d_session* s = NULL;

    for (i = 0; i < N * N; ++i) {
        rho[i] = 1000.0f; mu[i] = 1.0e9f; l2m[i] = 4.0e9f; lam[i] = 2.0e9f;
    }
    for (i = 0; i < N; ++i) { dp[i] = 3.0e9f; dx[i] = dxh[i] = dz[i] = dzh[i] = 0.0f; }
    CHECK2(seis2d_generate_ricker(wavelet, NT, 1.0e-4f, 200.0f, 0.005f));
    seis2d_stencil_weights(w);
    c.NX = N; c.NZ = N; c.total_grid = N * N; c.h = 1.0f; c.dt = 1.0e-4f; c.nt = NT; c.npml = 16;
    c.snap_spacenum = 1; c.flag_type = 1;
    c.rho.data = rho; c.rho.size = N * N; c.mu.data = mu; c.mu.size = N * N;
    c.lambda.data = lam; c.lambda.size = N * N; c.lambda2mu.data = l2m; c.lambda2mu.size = N * N;
    c.dp_flat.data = dp; c.dp_flat.size = N;
    c.dx.data = dx; c.dx.size = N; c.dx_half.data = dxh; c.dx_half.size = N;
    c.dz.data = dz; c.dz.size = N; c.dz_half.data = dzh; c.dz_half.size = N;
    c.c1_h = (float)w[0]; c.c2_h = (float)w[1]; c.c3_h = (float)w[2]; c.c4_h = (float)w[3];
    c.src_idx = (N / 2) * N + N / 2; c.src_z_idx = N / 2;
    c.wavelet.data = wavelet; c.wavelet.size = NT;
    c.src_angle = 0.0f; c.src_type = 0; c.src_amp = 1.0f;
    c.num_rcv = 1; c.rcv_grid_idx.data = &rcv; c.rcv_grid_idx.size = 1; c.upFlag = 0;
    CHECK2(seis2d_initialize(&s, &c));
    CHECK2(seis2d_gather_begin(s, 0, 1, NT));
    CHECK2(seis2d_run_steps(s, 0, NT, &c, -1));
    CHECK2(seis2d_gather_fetch(s, vx, vz, NT, &taken));
    *traceNorm = taken == NT ? norm(vz, NT) : -1.0;
    seis2d_release(s);
    return 0;
}

int main(int argc, char** argv) {
    double g3 = 0.0, t2 = 0.0;
    int exact = 0, rc;
    (void)argv;
    if (argc > 1) {
        /* Link check only: the library answers a host-only call. */
        printf("abi %d %d\n", seis3d_abi_version(), seis2d_abi_version());
        return 0;
    }
    rc = shot3d(&g3, &exact);
    if (rc) return rc;
    rc = shot2d(&t2);
    if (rc) return rc;
    printf("gather3d %.9e restart %d trace2d %.9e\n", g3, exact, t2);
    return 0;
}
