// ref_driver.cu -- project-written driver for building the UNMODIFIED
// reference single-GPU library (keita-akutagawa/ResistiveMHD_GPU,
// ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_{periodicXY,symmetricXY})
// as a test oracle and CPU/GPU baseline.  TEST INFRASTRUCTURE ONLY.
//
// The reference library is a set of sources that expect the user's driver to
// supply (see lib .../const.hpp:4-49 and flux_solver.hpp:23-29):
//   * link-time globals (EPS, dx, nx, ..., eta) and their __constant__ mirrors;
//   * ResistiveMHD2D::initializeU();
//   * FluxSolver::addResistiveTermToFluxF/G (the resistive flux hook).
// This file supplies them in the pattern of the reference's example drivers
// (ResistiveMHD_singleGPU_thrust/examples2D/plasmoid/main_plasmoid.cu:15-82,
// 132-290), with the grid read from the environment at static-init time so
// one binary serves every size, the initial state read from a file, and eta
// either uniform or read from a cell-centred table.
//
// Built twice by oracle/build_ref.py: with nvcc for sm_100a (GPU reference)
// and with g++ -fopenmp against Thrust's OMP backend (host reference), where
// REF_HOST_BUILD is defined and the launch macro below runs blocks on host
// threads.
//
// Usage:  <binary> in_state out_state n_warmup n_timed [dts_out]
// Environment: REF_NX REF_NY REF_DX REF_DY REF_GAMMA REF_CFL REF_EPS REF_ETA
//              [REF_ETA_TABLE=path to nx*ny doubles]
// Prints one JSON line with the timing of the n_timed steps: host wall clock
// ("seconds") and, in the GPU build, CUDA events on the legacy default stream
// around them ("event_seconds"; -1 in the host build).

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "const.hpp"
#include "resistiveMHD_2D.hpp"

#ifdef REF_HOST_BUILD
#include <omp.h>
#define REF_LAUNCH(kernel, grid, block, ...) host_launch((grid), (block), [&]() { kernel(__VA_ARGS__); })
#else
#define REF_LAUNCH(kernel, grid, block, ...) kernel<<<(grid), (block)>>>(__VA_ARGS__)
#endif

static double ref_env_double(const char *name, double fallback)
{
    const char *s = std::getenv(name);
    return s ? std::strtod(s, nullptr) : fallback;
}
static int ref_env_int(const char *name, int fallback)
{
    const char *s = std::getenv(name);
    return s ? std::atoi(s) : fallback;
}

// ---- globals declared extern by the library's const.hpp ----
const double EPS = ref_env_double("REF_EPS", 1e-20);
const double PI = 3.141592653589793;

const double dx = ref_env_double("REF_DX", 1.0);
const double xmin = 0.0;
const int nx = ref_env_int("REF_NX", 16);
const double xmax = nx * dx;

const double dy = ref_env_double("REF_DY", 1.0);
const double ymin = 0.0;
const int ny = ref_env_int("REF_NY", 16);
const double ymax = ny * dy;

const double CFL = ref_env_double("REF_CFL", 0.4);
const double gamma_mhd = ref_env_double("REF_GAMMA", 5.0 / 3.0);

double dt = 0.0;
const int totalStep = 0;
double totalTime = 0.0;
double eta = ref_env_double("REF_ETA", 0.0);

__constant__ double device_EPS;
__constant__ double device_PI;
__constant__ double device_dx;
__constant__ double device_xmin;
__constant__ double device_xmax;
__constant__ int device_nx;
__constant__ double device_dy;
__constant__ double device_ymin;
__constant__ double device_ymax;
__constant__ int device_ny;
__constant__ double device_CFL;
__constant__ double device_gamma_mhd;
__device__ double device_dt;
__device__ double device_eta;

// eta for the resistive hook: uniform value, or a cell-centred table.
__constant__ double device_eta_uniform;
__device__ const double *device_eta_table;

static std::vector<double> g_initial_state;

__device__ inline double driverEta(int i, int j)
{
    return device_eta_table ? device_eta_table[j + i * device_ny] : device_eta_uniform;
}

void ResistiveMHD2D::initializeU()
{
    thrust::host_vector<ConservationParameter> h(nx * ny);
    for (int k = 0; k < nx * ny; ++k) {
        const double *c = &g_initial_state[8 * (size_t)k];
        h[k].rho = c[0]; h[k].rhoU = c[1]; h[k].rhoV = c[2]; h[k].rhoW = c[3];
        h[k].bX = c[4]; h[k].bY = c[5]; h[k].bZ = c[6]; h[k].e = c[7];
    }
    U = h;
#ifdef REF_SYMMETRIC
    boundary.symmetricBoundaryX2nd(U);
    boundary.symmetricBoundaryY2nd(U);
#else
    boundary.periodicBoundaryX2nd(U);
    boundary.periodicBoundaryY2nd(U);
#endif
}

// Resistive flux hooks: the same arithmetic as the example drivers'
// addResistiveTermToFluxF/G_kernel (examples2D/plasmoid/main_plasmoid.cu:175-290),
// with eta sampled at cell centres (i, j) and (i+1, j) / (i, j+1).
__global__ void refResistiveF_kernel(const ConservationParameter *U, Flux *flux)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if ((0 < i) && (i < device_nx - 2) && (0 < j) && (j < device_ny - 2)) {
        const int n = device_ny;
        double a, b, e0, e1;
        a = -(U[j + (i + 1) * n].bZ - U[j + (i - 1) * n].bZ) / (2.0 * device_dx);
        b = (U[j + (i + 1) * n].bY - U[j + (i - 1) * n].bY) / (2.0 * device_dx)
          - (U[j + 1 + i * n].bX - U[j - 1 + i * n].bX) / (2.0 * device_dy);
        e0 = driverEta(i, j);
        double eJY0 = e0 * a, eJZ0 = e0 * b;
        double eJYBZ0 = eJY0 * U[j + i * n].bZ, eJZBY0 = eJZ0 * U[j + i * n].bY;
        a = -(U[j + (i + 2) * n].bZ - U[j + i * n].bZ) / (2.0 * device_dx);
        b = (U[j + (i + 2) * n].bY - U[j + i * n].bY) / (2.0 * device_dx)
          - (U[j + 1 + (i + 1) * n].bX - U[j - 1 + (i + 1) * n].bX) / (2.0 * device_dy);
        e1 = driverEta(i + 1, j);
        double eJY1 = e1 * a, eJZ1 = e1 * b;
        double eJYBZ1 = eJY1 * U[j + (i + 1) * n].bZ, eJZBY1 = eJZ1 * U[j + (i + 1) * n].bY;
        flux[j + i * n].f5 -= 0.5 * (eJZ0 + eJZ1);
        flux[j + i * n].f6 += 0.5 * (eJY0 + eJY1);
        flux[j + i * n].f7 += 0.5 * (eJYBZ0 + eJYBZ1) - 0.5 * (eJZBY0 + eJZBY1);
    }
}

__global__ void refResistiveG_kernel(const ConservationParameter *U, Flux *flux)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if ((0 < i) && (i < device_nx - 2) && (0 < j) && (j < device_ny - 2)) {
        const int n = device_ny;
        double a, b, e0, e1;
        a = (U[j + 1 + i * n].bZ - U[j - 1 + i * n].bZ) / (2.0 * device_dy);
        b = (U[j + (i + 1) * n].bY - U[j + (i - 1) * n].bY) / (2.0 * device_dx)
          - (U[j + 1 + i * n].bX - U[j - 1 + i * n].bX) / (2.0 * device_dy);
        e0 = driverEta(i, j);
        double eJX0 = e0 * a, eJZ0 = e0 * b;
        double eJXBZ0 = eJX0 * U[j + i * n].bZ, eJZBX0 = eJZ0 * U[j + i * n].bX;
        a = (U[j + 2 + i * n].bZ - U[j + i * n].bZ) / (2.0 * device_dy);
        b = (U[j + 1 + (i + 1) * n].bY - U[j + 1 + (i - 1) * n].bY) / (2.0 * device_dx)
          - (U[j + 2 + i * n].bX - U[j + i * n].bX) / (2.0 * device_dy);
        e1 = driverEta(i, j + 1);
        double eJX1 = e1 * a, eJZ1 = e1 * b;
        double eJXBZ1 = eJX1 * U[j + 1 + i * n].bZ, eJZBX1 = eJZ1 * U[j + 1 + i * n].bX;
        flux[j + i * n].f4 += 0.5 * (eJZ0 + eJZ1);
        flux[j + i * n].f6 -= 0.5 * (eJX0 + eJX1);
        flux[j + i * n].f7 += 0.5 * (eJZBX0 + eJZBX1) - 0.5 * (eJXBZ0 + eJXBZ1);
    }
}

void FluxSolver::addResistiveTermToFluxF(const thrust::device_vector<ConservationParameter> &U)
{
    dim3 threadsPerBlock(16, 16);
    dim3 blocksPerGrid((nx + threadsPerBlock.x - 1) / threadsPerBlock.x,
                       (ny + threadsPerBlock.y - 1) / threadsPerBlock.y);
    REF_LAUNCH(refResistiveF_kernel, blocksPerGrid, threadsPerBlock,
               thrust::raw_pointer_cast(U.data()), thrust::raw_pointer_cast(flux.data()));
    cudaDeviceSynchronize();
}

void FluxSolver::addResistiveTermToFluxG(const thrust::device_vector<ConservationParameter> &U)
{
    dim3 threadsPerBlock(16, 16);
    dim3 blocksPerGrid((nx + threadsPerBlock.x - 1) / threadsPerBlock.x,
                       (ny + threadsPerBlock.y - 1) / threadsPerBlock.y);
    REF_LAUNCH(refResistiveG_kernel, blocksPerGrid, threadsPerBlock,
               thrust::raw_pointer_cast(U.data()), thrust::raw_pointer_cast(flux.data()));
    cudaDeviceSynchronize();
}

static bool read_doubles(const char *path, std::vector<double> &out, size_t n)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    out.resize(n);
    size_t got = std::fread(out.data(), sizeof(double), n, f);
    std::fclose(f);
    return got == n;
}

int main(int argc, char **argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s in_state out_state n_warmup n_timed [dts_out]\n", argv[0]);
        return 2;
    }
    const size_t ncell = (size_t)nx * ny;
    if (!read_doubles(argv[1], g_initial_state, 8 * ncell)) {
        std::fprintf(stderr, "cannot read %zu cells from %s\n", ncell, argv[1]);
        return 2;
    }
    const int nwarm = std::atoi(argv[3]);
    const int ntimed = std::atoi(argv[4]);

    initializeDeviceConstants();
    double etaU = eta;
    cudaMemcpyToSymbol(device_eta_uniform, &etaU, sizeof(double));
    std::vector<double> etaTab;
    const double *etaTabPtr = nullptr;
    const char *etaPath = std::getenv("REF_ETA_TABLE");
#ifndef REF_HOST_BUILD
    double *etaDev = nullptr;
#endif
    if (etaPath && *etaPath) {
        if (!read_doubles(etaPath, etaTab, ncell)) {
            std::fprintf(stderr, "cannot read eta table %s\n", etaPath);
            return 2;
        }
#ifdef REF_HOST_BUILD
        etaTabPtr = etaTab.data();
#else
        cudaMalloc(&etaDev, ncell * sizeof(double));
        cudaMemcpy(etaDev, etaTab.data(), ncell * sizeof(double), cudaMemcpyHostToDevice);
        etaTabPtr = etaDev;
#endif
    }
    cudaMemcpyToSymbol(device_eta_table, &etaTabPtr, sizeof(etaTabPtr));

    ResistiveMHD2D solver;
    solver.initializeU();

    std::vector<double> dts;
    int crashedAt = -1;
    auto run = [&](int nsteps) {
        for (int s = 0; s < nsteps && crashedAt < 0; ++s) {
            solver.oneStepRK2();
            dts.push_back(dt);
            if (solver.checkCalculationIsCrashed()) crashedAt = (int)dts.size() - 1;
            totalTime += dt;
        }
    };
    run(nwarm);
#ifndef REF_HOST_BUILD
    cudaDeviceSynchronize();
    // device-side time of the timed steps: events on the legacy default
    // stream, which every launch, copy and synchronisation of the reference
    // library uses
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, 0);
#endif
    auto t0 = std::chrono::steady_clock::now();
    run(ntimed);
#ifndef REF_HOST_BUILD
    cudaEventRecord(ev1, 0);
    cudaDeviceSynchronize();
    float eventMs = 0.0f;
    cudaEventElapsedTime(&eventMs, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    const double eventSecs = 1e-3 * eventMs;
#else
    const double eventSecs = -1.0;
#endif
    auto t1 = std::chrono::steady_clock::now();
    double secs = std::chrono::duration<double>(t1 - t0).count();

    thrust::device_vector<ConservationParameter> Ud = solver.getU();
    thrust::host_vector<ConservationParameter> Uh = Ud;
    std::vector<double> out(8 * ncell);
    for (size_t k = 0; k < ncell; ++k) {
        double *c = &out[8 * k];
        c[0] = Uh[k].rho; c[1] = Uh[k].rhoU; c[2] = Uh[k].rhoV; c[3] = Uh[k].rhoW;
        c[4] = Uh[k].bX; c[5] = Uh[k].bY; c[6] = Uh[k].bZ; c[7] = Uh[k].e;
    }
    FILE *f = std::fopen(argv[2], "wb");
    if (!f) return 3;
    std::fwrite(out.data(), sizeof(double), out.size(), f);
    std::fclose(f);
    if (argc > 5) {
        FILE *g = std::fopen(argv[5], "wb");
        if (!g) return 3;
        std::fwrite(dts.data(), sizeof(double), dts.size(), g);
        std::fclose(g);
    }
#ifdef REF_HOST_BUILD
    int threads = omp_get_max_threads();
    const char *kind = "host-omp";
#else
    int threads = 0;
    const char *kind = "gpu";
#endif
    std::printf("{\"kind\": \"%s\", \"nx\": %d, \"ny\": %d, \"warmup\": %d, \"steps\": %d, "
                "\"seconds\": %.9g, \"event_seconds\": %.9g, \"threads\": %d, \"crashed_at\": %d, "
                "\"total_time\": %.17g}\n",
                kind, nx, ny, nwarm, ntimed, secs, eventSecs, threads, crashedAt, totalTime);
    return 0;
}
