// mc_driver.cu -- project-written driver for building parts of the UNMODIFIED
// multi-GPU library of keita-akutagawa/ResistiveMHD_GPU
// (ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU: const.cu, ct.cu,
// boundary.cu, mpi.cu, sign.cu) for the host, on one rank, as a checker of
// this project's restatements of its CT-Contact EMF and its walls.
// TEST INFRASTRUCTURE ONLY.  Built by oracle/build_ref.py with g++ against
// Thrust's OpenMP backend, oracle/ref_host_shim.h and the single-rank
// oracle/mpi_stub/mpi.h.
//
// The library expects the user's driver to supply the link-time globals of
// its const.hpp, device_eta and getEta (as ResistiveMHD_multiGPU_cuda/
// plasmoid/main_plasmoid.cu:15-90 does); here the grid comes from the
// environment at static-init time and eta from a cell-centred table or a
// uniform value.
//
// Usage:
//   mc_driver boundary <pair> in_state out_state
//       pair: periodic_periodic | periodic_wall | periodic_zerogradient | flare_wall
//       Runs the ghost fill of the matching step variant of the library's
//       resistiveMHD2D.cu: sendrecv_U (on one rank: the periodic copies in x,
//       then y) followed by the x and y wall functions
//       (oneStepRK2 :216-219, oneStepRK2_periodicXWallY :293-296,
//        oneStepRK2_periodicXSymmetricY :372-375, oneStepRK2_flareXWallY :449-452).
//   mc_driver ct in_dir out_state
//       in_dir holds u_old, f_old, g_old, u_now, f_now, g_now (nx*ny*8 doubles
//       each, the state and flux records), bx_old, by_old (nx*ny doubles);
//       runs CT::setOldFlux2D(f_old, g_old, u_old), CT::setNowFlux2D(f_now,
//       g_now, u_now) and CT::divBClean(bx_old, by_old, U = u_now) with
//       device_dt = MC_DT and writes U.
// Environment: REF_NX REF_NY (cells incl. 3 ghost layers per side), REF_DX
//              REF_DY REF_GAMMA REF_EPS REF_ETA [REF_ETA_TABLE] MC_DT.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "boundary.hpp"
#include "const.hpp"
#include "ct.hpp"
#include "mpi.hpp"

static double mc_env_double(const char *name, double fallback)
{
    const char *s = std::getenv(name);
    return s ? std::strtod(s, nullptr) : fallback;
}
static int mc_env_int(const char *name, int fallback)
{
    const char *s = std::getenv(name);
    return s ? std::atoi(s) : fallback;
}

// ---- globals declared extern by the library's const.hpp; nx, ny count the
// interior cells (the library adds its buffer of 3 per side) ----
const double EPS = mc_env_double("REF_EPS", 1e-20);
const double PI = 3.141592653589793;
const double dx = mc_env_double("REF_DX", 1.0);
const double xmin = 0.0;
const int nx = mc_env_int("REF_NX", 16) - 6;
const double xmax = nx * dx;
const double dy = mc_env_double("REF_DY", 1.0);
const double ymin = 0.0;
const int ny = mc_env_int("REF_NY", 16) - 6;
const double ymax = ny * dy;
const double CFL = 0.4;
const double gamma_mhd = mc_env_double("REF_GAMMA", 5.0 / 3.0);
double dt = mc_env_double("MC_DT", 0.0);
const int totalStep = 0;
double totalTime = 0.0;

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

static double g_eta_uniform = mc_env_double("REF_ETA", 0.0);
static std::vector<double> g_eta_table;

// The library samples eta at (i dx, j dy) of array cell (i, j) (ct.cu:42-56);
// the position is turned back into the cell to read a cell-centred table.
__device__ double getEta(double &xPosition, double &yPosition)
{
    if (g_eta_table.empty()) return g_eta_uniform;
    const long i = std::lround(xPosition / dx), j = std::lround(yPosition / dy);
    return g_eta_table[(size_t)(j + i * (ny + 6))];
}

static bool read_doubles(const std::string &path, std::vector<double> &out, size_t n)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out.resize(n);
    const size_t got = std::fread(out.data(), sizeof(double), n, f);
    std::fclose(f);
    return got == n;
}

template <class Rec> static thrust::device_vector<Rec> to_records(const std::vector<double> &v)
{
    static_assert(sizeof(Rec) == 8 * sizeof(double), "8-double records");
    thrust::host_vector<Rec> h(v.size() / 8);
    std::memcpy(thrust::raw_pointer_cast(h.data()), v.data(), v.size() * sizeof(double));
    return thrust::device_vector<Rec>(h);
}

static bool write_state(const char *path, const thrust::device_vector<ConservationParameter> &U)
{
    thrust::host_vector<ConservationParameter> h = U;
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    std::fwrite(thrust::raw_pointer_cast(h.data()), sizeof(ConservationParameter), h.size(), f);
    std::fclose(f);
    return true;
}

int main(int argc, char **argv)
{
    if (argc < 4 || (std::string(argv[1]) == "boundary" && argc < 5)) {
        std::fprintf(stderr, "usage: %s boundary <pair> in out | %s ct in_dir out\n", argv[0], argv[0]);
        return 2;
    }
    const size_t ncell = (size_t)(nx + 6) * (ny + 6);
    initializeDeviceConstants();
    const char *etaPath = std::getenv("REF_ETA_TABLE");
    if (etaPath && *etaPath && !read_doubles(etaPath, g_eta_table, ncell)) {
        std::fprintf(stderr, "cannot read eta table %s\n", etaPath);
        return 2;
    }
    MPIInfo info;
    setupInfo(info, 3);
    const std::string mode = argv[1];
    if (mode == "boundary") {
        std::vector<double> in;
        if (!read_doubles(argv[3], in, 8 * ncell)) return 2;
        thrust::device_vector<ConservationParameter> U = to_records<ConservationParameter>(in);
        Boundary boundary(info);
        const std::string pair = argv[2];
        sendrecv_U(U, info);
        if (pair == "periodic_periodic") {
            boundary.periodicBoundaryX2nd_U(U);
            boundary.periodicBoundaryY2nd_U(U);
        } else if (pair == "periodic_wall") {
            boundary.periodicBoundaryX2nd_U(U);
            boundary.wallBoundaryY2nd_U(U);
        } else if (pair == "periodic_zerogradient") {
            boundary.periodicBoundaryX2nd_U(U);
            boundary.symmetricBoundaryY2nd_U(U);
        } else if (pair == "flare_wall") {
            boundary.flareBoundaryX2nd_U(U);
            boundary.wallBoundaryY2nd_U(U);
        } else {
            std::fprintf(stderr, "unknown pair %s\n", pair.c_str());
            return 2;
        }
        return write_state(argv[4], U) ? 0 : 3;
    }
    if (mode == "ct") {
        const std::string d = std::string(argv[2]) + "/";
        std::vector<double> uo, fo, go, un, fn, gn, bxo, byo;
        if (!read_doubles(d + "u_old", uo, 8 * ncell) || !read_doubles(d + "f_old", fo, 8 * ncell) ||
            !read_doubles(d + "g_old", go, 8 * ncell) || !read_doubles(d + "u_now", un, 8 * ncell) ||
            !read_doubles(d + "f_now", fn, 8 * ncell) || !read_doubles(d + "g_now", gn, 8 * ncell) ||
            !read_doubles(d + "bx_old", bxo, ncell) || !read_doubles(d + "by_old", byo, ncell)) {
            std::fprintf(stderr, "cannot read the CT inputs from %s\n", argv[2]);
            return 2;
        }
        CT ct(info);
        ct.setOldFlux2D(to_records<Flux>(fo), to_records<Flux>(go), to_records<ConservationParameter>(uo));
        ct.setNowFlux2D(to_records<Flux>(fn), to_records<Flux>(gn), to_records<ConservationParameter>(un));
        thrust::device_vector<ConservationParameter> U = to_records<ConservationParameter>(un);
        thrust::device_vector<double> bXOld(bxo.begin(), bxo.end()), bYOld(byo.begin(), byo.end());
        ct.divBClean(bXOld, bYOld, U);
        return write_state(argv[3], U) ? 0 : 3;
    }
    std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}
